/*
 * b200md.h -- C ABI of the B200 short-range MD engine (libb200md.so).
 *
 * One context (b200_ctx) holds one periodic orthogonal box of atoms resident
 * in the GPU's memory, its cell-sorted neighbor list and its pair potential.
 * A LAMMPS Pair/Fix subclass (lammps_b200/lammps/) or any other host drives
 * it with plain pointers and sizes; no C++ or torch types cross the boundary.
 *
 * Reference interfaces replaced (LAMMPS 8 Aug 2014, paths inside the
 * reference project):
 *   - the GPU package's C ABI for pair styles: ljl_gpu_init / ljl_gpu_compute /
 *     ljl_gpu_compute_n / ljl_gpu_clear (lib/gpu/lal_lj_ext.cpp:25-141, bound
 *     in src/GPU/pair_lj_cut_gpu.cpp:42-65) and eam_gpu_* with
 *     eam_gpu_compute_force (lib/gpu/lal_eam_ext.cpp:30,122,133);
 *   - the per-step callbacks a Pair and a Fix implement: Pair::compute
 *     (src/pair.h:135), FixNVE::initial_integrate / final_integrate
 *     (src/fix_nve.cpp:65-142), Neighbor::build (src/neighbor.cpp:1380) and
 *     the NeighList arrays (src/neigh_list.h:35-39).
 *
 * Conventions
 *   - Every entry point returns an int status: 0 (B200_OK) or a negative
 *     B200_ERR_* code; b200_last_error() gives the message.  Nothing throws
 *     across the ABI and no kernel traps: device-side failures set a status
 *     word that the host reads (as src/GPU/gpu_extra.h:26-64 maps the GPU
 *     package's negative codes to error->all).
 *   - Per-type tables use LAMMPS's 1-based layout flattened row-major:
 *     an (ntypes+1) x (ntypes+1) array t has t[i*(ntypes+1)+j] for types
 *     i,j in 1..ntypes; per-type vectors have ntypes+1 entries.
 *   - Per-atom arrays are in the caller's order (the order of the last
 *     b200_upload_atoms), xyz interleaved: x[3*i+0..2].
 *   - Calls on one context are stream-ordered on that context's CUDA stream
 *     and must come from one host thread at a time.
 */
#ifndef B200MD_H
#define B200MD_H

#ifdef __cplusplus
extern "C" {
#endif

#define B200MD_ABI_VERSION 1

typedef struct b200_ctx b200_ctx;

enum b200_status {
  B200_OK = 0,
  B200_ERR_ARG = -1,            /* bad argument (error->all "Illegal ...") */
  B200_ERR_CUDA = -2,           /* CUDA runtime error */
  B200_ERR_NOMEM = -3,          /* device allocation failed */
  B200_ERR_STATE = -4,          /* call out of order (e.g. compute before atoms) */
  B200_ERR_NEIGH_OVERFLOW = -5, /* "Neighbor list overflow, boost neigh_modify one" */
  B200_ERR_BOX = -6,            /* box edge not larger than the ghost cutoff (mixed form:
                                   not longer than twice the list cutoff) */
  B200_ERR_LOST_ATOMS = -7,     /* non-finite coordinate or atom beyond one box image */
  B200_ERR_TIMEOUT = -8         /* a bounded device wait expired */
};

enum b200_precision {
  B200_PREC_FP64 = 0,  /* all pair arithmetic in FP64: the drop-in form */
  B200_PREC_MIXED = 1  /* FP32 pair math on separations from 32-bit fixed-point
                          coordinates (box edges must exceed twice the list
                          cutoff), FP64 positions, per-atom force sums and
                          global sums */
};

enum b200_pair_style { B200_PAIR_NONE = 0, B200_PAIR_LJ_CUT = 1, B200_PAIR_EAM = 2 };

/* ---- context ------------------------------------------------------------ */

/* Create a context on CUDA device `device` (replaces ljl_gpu_init's device
   and precision selection, lib/gpu/lal_lj_ext.cpp:25-97). */
int b200_create(int device, int precision, b200_ctx **out);
/* Free every device buffer of the context (ljl_gpu_clear,
   lib/gpu/lal_lj_ext.cpp:101-103). */
int b200_destroy(b200_ctx *ctx);
/* Message of the last failing call on this context (or of b200_create). */
const char *b200_last_error(const b200_ctx *ctx);
int b200_abi_version(void);
/* Device bytes held by the context (ljl_gpu_bytes, lib/gpu/lal_lj_ext.cpp:139). */
long long b200_bytes(const b200_ctx *ctx);

/* ---- settings ----------------------------------------------------------- */

/* Orthogonal periodic box [lo,hi) in every dimension (Domain boxlo/boxhi,
   src/domain.cpp:213-217). */
int b200_set_box(b200_ctx *ctx, const double lo[3], const double hi[3]);
/* `neighbor skin bin` + `neigh_modify every/delay/check/one`
   (src/neighbor.cpp:1731-1790).  one > 0 is a hard per-atom limit: a list
   longer than that fails with B200_ERR_NEIGH_OVERFLOW, as the reference's
   "Neighbor list overflow, boost neigh_modify one".  one == 0 sizes the list
   from the density, one < 0 starts at -one entries per atom; in both cases
   the list grows when needed (b200_run replays a chunk that overflowed). */
int b200_set_neighbor(b200_ctx *ctx, double skin, int every, int delay, int check, int one);
/* Per-type masses, mass[1..ntypes] (Atom::mass). */
int b200_set_mass(b200_ctx *ctx, int ntypes, const double *mass);
/* pair_style lj/cut tables after PairLJCut::init_one
   (src/pair_lj_cut.cpp:545-602): cutsq, lj1..lj4, offset. */
int b200_set_lj(b200_ctx *ctx, int ntypes, const double *cutsq, const double *lj1,
                const double *lj2, const double *lj3, const double *lj4, const double *offset);
/* pair_style eam / eam/alloy / eam/fs spline tables after PairEAM::file2array
   and array2spline (src/MANYBODY/pair_eam.cpp:488-719): 7 coefficients per
   knot, knots 0..n (row 0 unused), tables back to back:
     frho_spline[nfrho][nrho+1][7], rhor_spline[nrhor][nr+1][7],
     z2r_spline[nz2r][nr+1][7];
   type2frho[ntypes+1], type2rhor and type2z2r [(ntypes+1)^2]. */
int b200_set_eam(b200_ctx *ctx, int ntypes, int nrho, double drho, int nr, double dr,
                 double rhomax, double cutmax, int nfrho, const double *frho_spline, int nrhor,
                 const double *rhor_spline, int nz2r, const double *z2r_spline,
                 const int *type2frho, const int *type2rhor, const int *type2z2r);

/* ---- atoms ----------------------------------------------------------------- */

/* Copy n atoms to the device (AtomVec x, v, type, tag; ljl_gpu_compute's x
   upload, lib/gpu/lal_base_atomic.cpp:176-241).  v may be NULL (zero).  The
   arrays may be host or device memory (unified addressing), as may the
   destinations of b200_download_atoms and the per-atom arrays of
   b200_pair_compute. */
int b200_upload_atoms(b200_ctx *ctx, int n, const double *x, const double *v, const int *type,
                      const int *tag);
/* Copy positions, velocities, forces and image flags back, in the caller's
   order (NULL pointers are skipped; image is 3 ints per atom). */
int b200_download_atoms(b200_ctx *ctx, double *x, double *v, double *f, int *image);
int b200_natoms(const b200_ctx *ctx);

/* Overlapped transfers, for a caller that runs one atom set after another:
   each set's host copies overlap the device work of the set before it, as the
   reference's GPU library overlaps its asynchronous position upload and
   answer download with the host's work (Atom::add_x_data,
   lib/gpu/lal_atom.h:282-297; Answer::copy_answers, lib/gpu/lal_answer.cpp:140-162).
   The context copies on two streams of its own (one per direction) through
   device buffers of its own; page-locked host memory lets the copies run
   beside the kernels.

   b200_stage_atoms starts copying an atom set (the arguments of
   b200_upload_atoms, without tag) into one of two device slots and returns
   without waiting.  The host arrays must stay unchanged until
   b200_set_staged_atoms has taken the set.  At most two sets wait at a time
   (B200_ERR_STATE beyond that).
   b200_set_staged_atoms makes the oldest staged set the context's atoms:
   b200_upload_atoms from the slot, once its copy has arrived; its types are
   checked on the device (B200_ERR_ARG for a type outside 1..ntypes).
   b200_download_atoms_async forms the arrays of b200_download_atoms on the
   device now and copies them to the host arrays while later work runs; they
   are valid after b200_wait_transfers, which waits for every copy started
   by either call. */
int b200_stage_atoms(b200_ctx *ctx, int n, const double *x, const double *v, const int *type);
int b200_set_staged_atoms(b200_ctx *ctx);
int b200_download_atoms_async(b200_ctx *ctx, double *x, double *v, double *f, int *image);
int b200_wait_transfers(b200_ctx *ctx);
/* New positions x[3n] (caller order, host or device memory) for the atoms of
   the last upload, keeping their cells and the neighbor list of the last
   build: the per-step position refresh of a Pair::compute between
   reneighborings, when the host integrates and Neighbor::decide
   (src/neighbor.cpp:1294-1320) has not asked for a rebuild.  Like the
   reference, forces use the list as built; the caller rebuilds (upload +
   b200_neigh_build) on its reneighbor steps. */
int b200_update_positions(b200_ctx *ctx, const double *x);

/* Column groups of b200_gather. */
enum b200_field {
  B200_FIELD_X = 1,     /* x y z */
  B200_FIELD_V = 2,     /* vx vy vz */
  B200_FIELD_F = 4,     /* fx fy fz */
  B200_FIELD_IMAGE = 8  /* box crossings since the upload, ix iy iz (as doubles) */
};
/* The per-atom columns a dump writes, straight from the device: the
   per-atom part of DumpCustom::pack (src/dump_custom.cpp:913-961) without a
   download of the whole state.  Row r of out (host or device memory) holds
   the requested groups, in the order x, v, f, image, of atom idx[r] (caller
   index; host or device memory), or of atom r when idx is NULL; out has
   m * 3 * (number of groups) doubles.  An index outside [0, n) returns
   B200_ERR_ARG. */
int b200_gather(b200_ctx *ctx, int fields, int m, const int *idx, double *out);

/* ---- per-step entry points ------------------------------------------------- */

/* Domain::pbc + periodic images + cell counting sort + full neighbor list
   (Domain::pbc src/domain.cpp:478, CommBrick::borders src/comm_brick.cpp:696,
   Neighbor::build src/neighbor.cpp:1380). */
int b200_neigh_build(b200_ctx *ctx);
/* Pair::compute(eflag, vflag) (src/pair.h:135): forces on the device;
   eflag/vflag as Integrate::ev_set (src/integrate.cpp:114-149).  Energy and
   virial go to *eng and virial[6] when the global flags are set (NULL to keep
   them on the device), per-atom eatom[n] / vatom[6n] when the atom flags are
   set (NULL to skip). */
int b200_pair_compute(b200_ctx *ctx, int eflag, int vflag, double *eng, double virial[6],
                      double *eatom, double *vatom);
/* FixNVE::initial_integrate / final_integrate (src/fix_nve.cpp:65-142):
   dtv = dt, dtf = 0.5 dt ftm2v. */
int b200_nve_initial(b200_ctx *ctx, double dtv, double dtf);
int b200_nve_final(b200_ctx *ctx, double dtf);

/* Verlet::setup (src/verlet.cpp:88-142): wrap, build, forces at the current
   step with energy and virial.  Returns the thermo row of that step. */
int b200_setup(b200_ctx *ctx, double *row);
/* Verlet::run(nsteps) (src/verlet.cpp:207-309) with fix nve and the
   neighbor schedule of b200_set_neighbor; the atoms never leave the device.
   The host mirrors Neighbor::decide and reads the device's distance test
   back only on steps where `check yes` could rebuild.  Every `thermo_every`
   steps and at the last step a thermo row is recorded:
     row = {step, sum m v^2, eng_vdwl, virial[0..5]}  (9 doubles)
   from which the host forms Temp, E_pair, TotEng and Press exactly as
   ComputeTemp/ComputePressure do.  rows may be NULL; *nrows receives the
   number of rows recorded (at most maxrows are written). */
int b200_run(b200_ctx *ctx, int nsteps, double dt, double ftm2v, int thermo_every, double *rows,
             int maxrows, int *nrows);

/* ---- neighbor list and diagnostics ----------------------------------------- */

/* The half neighbor list that Neighbor::half_bin_newton
   (src/neigh_half_bin.cpp:285-419) builds from the same atoms and index
   order: per atom numneigh[n]; entries (jowner = caller index of the atom,
   jimage = (sx+1)+3(sy+1)+9(sz+1) periodic image) concatenated in atom
   order.  *total receives the entry count; at most cap entries are written. */
int b200_neigh_half(b200_ctx *ctx, int *numneigh, int *jowner, int *jimage, long long cap,
                    long long *total);
/* Full-list statistics: entries (2x the half-list count), builds since
   b200_setup (Neighbor::ncalls), dangerous builds (ndanger), the largest
   per-atom count and the list capacity per atom. */
int b200_neigh_stats(b200_ctx *ctx, long long *full_total, int *ncalls, int *ndanger,
                     int *maxneigh, int *capacity);
/* EAM density and embedding derivative of the last compute (PairEAM rho, fp). */
int b200_get_rho_fp(b200_ctx *ctx, double *rho, double *fp);

/* Launch shape of the pair kernels: threads per atom (1,2,4,8,16,32; 0 = chosen by
   the autotuner on the next b200_setup) and threads per block.  With 0, a box that
   steps through the one-launch step kernel (a single box, no ghosts) is searched
   once more between two steps, 50 steps into the first b200_run, on the evolved
   state; the search leaves positions, velocities and counters as it found them.
   Results are bit-reproducible at a fixed shape; two searched runs may pick
   different shapes, and then differ in the last bits of FP64 sums. */
int b200_set_launch(b200_ctx *ctx, int threads_per_atom, int block_size);
int b200_get_launch(const b200_ctx *ctx, int *threads_per_atom, int *block_size);
/* Phase timers of b200_run (the Timer categories of Verlet::run,
   src/timer.h:19-20, src/verlet.cpp:237-306), measured on the device with
   CUDA events recorded inside each step's graph.  Phases:
     0 fix nve initial half-step + rebuild decision
     1 neighbor rebuild (wrap, cell sort, list) -- near zero on steps without
     2 pair pass 1 (LJ force; EAM density + embedding)
     3 pair pass 2 (EAM force; zero for LJ)
     4 fix nve final half-step (+ kinetic energy and thermo row on output steps)
   b200_get_timing returns milliseconds summed over the timed steps.
   on = 2 times whole pieces instead, with the run's own step form kept
   (lj/cut forces and both half-steps in one launch): two stream events around
   each piece; phase 0 = initial half-steps at chunk starts, 1 = rebuilds,
   2 = forces with their half-steps; 3 and 4 stay zero. */
int b200_set_timing(b200_ctx *ctx, int on);
/* on = 1 (default): b200_run replays captured CUDA graphs of the step's
   pieces (initial half-step + decision, rebuild, forces + final half-step).
   on = 0: the same kernels launched one by one (for profilers and hosts
   that do not want graphs).  Both follow the same host-mirrored rebuild
   schedule and give identical results. */
int b200_set_graphs(b200_ctx *ctx, int on);
int b200_get_timing(b200_ctx *ctx, double phase_ms[5], long long *steps, int reset);
/* Device time of every step timed since the last reset (milliseconds, from
   the step's first phase event to its last; timing must be on): *count
   receives the number of steps, at most cap are written. */
int b200_get_step_times(b200_ctx *ctx, double *ms, int cap, int *count, int reset);
/* Kernel launches issued by the context since creation (for accounting);
   kernels replayed inside step graphs are counted per replay. */
long long b200_kernel_launches(const b200_ctx *ctx);
/* CUDA stream of the context, as a void* (cudaStream_t). */
void *b200_stream(const b200_ctx *ctx);

/* ---- spatial decomposition (one brick of a box per rank) ------------------- */

/* A rank's context holds the whole periodic box with its own atoms and, as
   ghosts, the atoms of other ranks within the ghost depth of its brick, at
   their own (unshifted) coordinates; the builder forms periodic images as for
   a single box.  These calls carry the per-rank parts of CommBrick and
   Neighbor::decide; the exchange between ranks is the caller's (NCCL or any
   transport).

   Mark the ghosts of the current atoms: ghost[i] != 0 for caller index i
   (upload order), n ints in host or device memory; NULL clears.  Ghosts are not
   integrated by b200_nve_initial / b200_nve_final, are left out of the
   distance check and of the kinetic energy, and get their positions from
   b200_halo_unpack.  Cleared by every b200_upload_atoms.  b200_run refuses a
   context with ghosts (it decides rebuilds alone; a decomposed box decides
   them across ranks).  The borders step, CommBrick::borders
   (src/comm_brick.cpp:696-864), is the caller's choice of ghosts. */
int b200_set_ghosts(b200_ctx *ctx, const int *ghost);
/* The local half of Neighbor::check_distance (src/neighbor.cpp:1322-1372):
   *moved = 1 if some owned atom moved more than half the skin since the last
   build, as tested by the b200_nve_initial calls since the last check (the
   flag is cleared).  The caller reduces it over ranks (MPI_Allreduce MAX,
   src/neighbor.cpp:1369).  Needs check yes (b200_set_neighbor). */
int b200_neigh_check(b200_ctx *ctx, int *moved);
/* CommBrick::forward_comm with AtomVecAtomic::pack_comm / unpack_comm
   (src/comm_brick.cpp:444-511, src/atom_vec_atomic.cpp:105-217), local
   halves.  idx[m] are caller indices and buf[3m] the coordinates, both
   DEVICE pointers on the context's device; the calls are ordered on the
   context's stream and return after it completes.  pack: buf[3i..3i+2] = x
   of atom idx[i].  unpack: x of atom idx[i] = buf[3i..3i+2].  An index
   outside [0, n) -- or, when ghosts are marked (b200_set_ghosts), an index
   of an owned atom -- is not written and the call returns B200_ERR_ARG. */
int b200_halo_pack(b200_ctx *ctx, int m, const int *idx, double *buf);
int b200_halo_unpack(b200_ctx *ctx, int m, const int *idx, const double *buf);

/* PairEAM::compute in two calls around the forward communication of F'(rho)
   (src/MANYBODY/pair_eam.cpp:160-232, then :237-303), for a context whose
   ghosts get F' from their owners -- the split of the GPU package's
   eam_gpu_compute / eam_gpu_compute_force with its fp_ptr
   (lib/gpu/lal_eam_ext.cpp:122,133).  b200_eam_density: rho, F'(rho) and the
   embedding energy of every atom (a ghost's F' is then overwritten by
   b200_eam_fp_unpack).  b200_eam_fp_pack / unpack: F' of the caller atoms
   idx[0..m) to / from buf[m] (DEVICE pointers; PairEAM::pack_forward_comm /
   unpack_forward_comm, src/MANYBODY/pair_eam.cpp:809-831); unpack writes
   ghosts only when ghosts are marked.  b200_eam_force: forces, with energy
   and virial as b200_pair_compute, completing the tallies of the density
   call; it must follow a b200_eam_density with the same eflag and vflag. */
int b200_eam_density(b200_ctx *ctx, int eflag, int vflag);
int b200_eam_fp_pack(b200_ctx *ctx, int m, const int *idx, double *buf);
int b200_eam_fp_unpack(b200_ctx *ctx, int m, const int *idx, const double *buf);
int b200_eam_force(b200_ctx *ctx, int eflag, int vflag, double *eng, double virial[6],
                   double *eatom, double *vatom);

/* ---- batched replicas ---------------------------------------------------- */

/* No counterpart in the reference (which runs one box per process): make the
   context hold nrep independent orthogonal periodic boxes, replica r with
   natoms[r] atoms in the box lo[3r..3r+2], hi[3r..3r+2] (Domain boxlo/boxhi
   per replica).  Replaces b200_set_box; the next b200_upload_atoms takes the
   replicas' atoms concatenated in replica order (sum natoms atoms).  All
   replicas share the pair style (lj/cut), masses, neighbor settings and
   timestep, and b200_setup / b200_run advance them together -- each kernel
   covers every replica, each atom and each cell tile knowing its own box.
   The thermo rows of b200_run then sum over all replicas; per-replica rows
   come from b200_replica_thermo. */
int b200_set_replicas(b200_ctx *ctx, int nrep, const int *natoms, const double *lo,
                      const double *hi);
int b200_replica_count(const b200_ctx *ctx);
/* Step form of a replica batch.  mode 1: a graph of kernels per MD step
   (the pair kernel over every replica, then the fused half-steps).  mode 2:
   one launch per MD step (between rebuilds and outputs): thread-block
   clusters of `cluster` CTAs of `block` threads, each cluster owning a fixed
   set of whole replicas balanced by atom count, compute their forces, meet at
   a cluster barrier, and apply the final half-step and the next initial
   half-step; the last CTA makes the rebuild decision.  `tpa` threads per
   atom.  mode 0 (default): the next b200_setup times the graph path and every
   one-launch shape (cluster 1/2/4, block 256/512, tpa 1/2/4; a nonzero
   argument fixes that value) and keeps the fastest.  Both forms give the same
   results bit for bit.  Applies from the next b200_setup. */
int b200_set_replica_step(b200_ctx *ctx, int mode, int cluster, int block, int tpa);
/* The form in use (*onelaunch 1 for the one-launch step) with its shape, and
   ms[0], ms[1]: the per-step device time of the graph path and of the best
   one-launch shape measured by the last tuning (0 when not measured). */
int b200_get_replica_step(const b200_ctx *ctx, int *onelaunch, int *cluster, int *block, int *tpa,
                          double *ms);
/* Per-replica thermo of the current positions and velocities (forces are
   recomputed with per-atom energy and virial): rows[9r..9r+8] =
   {natoms, sum m v^2, eng_vdwl, virial[0..5]}, from which Temp, E_pair and
   Press of replica r follow as for b200_run's rows. */
int b200_replica_thermo(b200_ctx *ctx, double *rows);

/* ---- differentiable force matching (pair_style lj/cut) ------------------- */

/* No counterpart in the reference: gradients of a force-matching loss for
   lj/cut with up to 4 atom types.  The context holds the atoms and the list
   (b200_set_lj with the cutoffs to use, b200_upload_atoms, b200_neigh_build).
   lj1, lj2 and cutsq are host (ntypes+1)^2 tables as in b200_set_lj;
   x, f, g and gx are DEVICE arrays of 3n doubles in the caller's atom order.
   Each call returns after its kernels have finished.

   Replace the positions (device array) and rebuild the list. */
int b200_adj_set_positions(b200_ctx *ctx, const double *x);
/* F_i = sum_j phi(r_ij) (x_i - x_j), phi = (lj1 r^-6 - lj2) r^-8 inside
   cutsq (PairLJCut::compute's pair force, src/pair_lj_cut.cpp:100-113);
   FP32 pair math with FP64 sums for a B200_PREC_MIXED context, FP64
   otherwise.  Each cutsq entry must lie within the list's cutoff. */
int b200_adj_forces(b200_ctx *ctx, const double *lj1, const double *lj2, const double *cutsq,
                    double *f);
/* Given g = dL/dF: gx = dL/dx (the Hessian-vector product of the forces
   with g) and glj1, glj2 = dL/dlj1, dL/dlj2 per type pair (host,
   (ntypes+1)^2; the cutoff itself is held fixed). */
int b200_adj_backward(b200_ctx *ctx, const double *lj1, const double *lj2, const double *cutsq,
                      const double *g, double *gx, double *glj1, double *glj2);

/* ---- allocation-free entry point -------------------------------------------- */

/* No counterpart in the reference.  Sum over n atoms of
   (vx^2 + vy^2 + vz^2) * mass[type[i]] -- the sum ComputeTemp::compute_scalar
   forms before scaling -- written to out[0], for callers that must not
   allocate device memory at the point of the call: code recording a CUDA
   graph by stream capture (where cudaMalloc is not allowed) or a host whose
   device memory belongs to another allocator.  No context is needed; v
   (3n doubles, xyz interleaved), type (n ints, each in 1..ntypes), mass
   (ntypes+1 doubles) and out are device pointers (an atom whose type lies
   outside 1..ntypes is not looked up in mass; it makes out[0] NaN, which the
   caller sees when it reads the result), and the call is ordered
   on `stream` (a cudaStream_t; NULL = the legacy default stream).  It
   allocates nothing: its reduction scratch is a fixed static device array
   (1184 block partials and a counter, about 9.5 KB per device) whose address
   is looked up on the first call on each device, so make that first call
   before any stream capture begins.  n is limited to the engine's atom limit
   (2^26 - 1) and ntypes to 8: larger values return B200_ERR_ARG.  All calls
   share the one scratch array, so calls that may overlap on the GPU (other
   streams, other host threads) race and must be serialised by the caller. */
int b200_kinetic_sum_noalloc(int n, const double *v, const int *type, const double *mass,
                             int ntypes, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
