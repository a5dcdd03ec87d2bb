// md_common.cuh -- shared device definitions of the B200 MD engine.
//
// Device-resident layout of one box (all arrays in cell-sorted order):
//   x4[i]      double4 (x, y, z, type)       -- FP64 positions, gathered per pair
//   v[3][n]    double SoA                     -- velocities
//   f[3][n]    double SoA                     -- forces (owner-summed; no ghosts)
//   xq[i]      int4 (x, y, z as 32-bit fixed-point fractions of the box edge,
//              type) -- mixed precision only (md_xq)
//   cell[i]    packed cell coordinates cx | cy<<10 | cz<<20 of the last build
//   nlist      neighbor list in int4 slabs (md_slab): bits 6..31 = neighbor
//              atom index, bits 0..5 = offset of the neighbor's cell from the
//              atom's cell, two bits per dimension (d+1 for d = -1,0,1).
// Periodic images are never stored: a neighbor in a wrapped cell is the owner
// atom plus the box shift implied by the offset code, so the reference's
// ghost atoms, forward_comm and reverse_comm disappear.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define MD_MAXTYPES 8
#define MD_TILE_CELLS 4    // cells along x owned by one neighbor-builder CTA
#define MD_ADJ_MAXTYPES 4  // types of the force-matching adjoint (16 type pairs)
#define MD_JBITS 26
#define MD_JMASK ((1u << MD_JBITS) - 1u)
#define MD_MAX_ATOMS ((int)MD_JMASK)
#define MD_CELLBITS 10
#define MD_MAX_CELLS_DIM (1 << MD_CELLBITS)

// status words in device memory (read by the host after a step or a run)
enum {
  ST_MAXNEIGH = 0,   // largest per-atom full-list count seen at the last build
  ST_LOST = 1,       // a coordinate was non-finite or beyond one box image
  ST_MOVED = 2,      // some atom moved more than half the skin (check yes)
  ST_REBUILD = 3,    // decision of the current step
  ST_AGO = 4,        // steps since the last build (Neighbor::ago)
  ST_NCALLS = 5,     // builds since setup (Neighbor::ncalls)
  ST_NDANGER = 6,    // dangerous builds (Neighbor::ndanger)
  ST_OVERFLOW = 7,   // a build exceeded the list capacity (sticky)
  ST_ROW = 8,        // thermo rows written by the device in this run
  ST_STEP_LO = 9,    // current timestep (low/high 32 bits)
  ST_STEP_HI = 10,
  ST_FORCE_BUILD = 11,  // rebuild on the next step regardless of the schedule
  ST_MAXSTAGE = 12,     // most atoms staged by one neighbor-builder tile since setup
  ST_HALO_BAD = 13,     // a halo pack/unpack index was outside [0, n)
  ST_BADTYPE = 14,      // 1 + index of an uploaded atom with a type outside [1, ntypes]
  ST_COUNT = 16
};

struct BoxGeom {
  double lo[3], hi[3], prd[3];
  double cinv[3];    // cells per unit length: ncell/prd
  double cs[3];      // cell edge prd/ncell
  double qinv[3];    // fixed-point units per unit length: 2^32/prd (md_xq)
  // length of one fixed-point unit, prd/2^32, as an FP32 pair hi + lo (a
  // single FP32 value would scale every separation by the same rounding
  // error); and 1/unit^2 the same way, for one unit in every dimension
  float qs[3], qs_lo[3];
  float q2inv, q2inv_lo;
  int qiso;          // the three edges are equal (one fixed-point unit)
  int ncell[3];
};

// Replica tables of a batched context: several independent periodic boxes
// advanced together in one set of device arrays.  The atoms of replica r
// always occupy the sorted indices [atom_start[r], atom_start[r+1]) (a
// rebuild only permutes atoms within their replica), and its cells the
// global cell indices [cell_base[r], cell_base[r] + ncells(r)).
struct Reps {
  const BoxGeom *box;      // per replica
  const int *rep_of_atom;  // per sorted atom index (fixed)
  const int *cell_base;    // per replica
  const int *tile_rep;     // per neighbor-builder tile
  const int *tile_base;    // per replica: its first builder tile
};

struct LJParamsDev {
  // (ntypes+1)^2 tables, row-major, as LAMMPS's 1-based arrays
  double cutsq[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  double lj1[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  double lj2[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  double lj3[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  double lj4[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  double offset[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
};

__host__ __device__ inline int md_cell_pack(int cx, int cy, int cz) {
  return cx | (cy << MD_CELLBITS) | (cz << (2 * MD_CELLBITS));
}
__host__ __device__ inline void md_cell_unpack(int c, int &cx, int &cy, int &cz) {
  cx = c & (MD_MAX_CELLS_DIM - 1);
  cy = (c >> MD_CELLBITS) & (MD_MAX_CELLS_DIM - 1);
  cz = c >> (2 * MD_CELLBITS);
}

// neighbor-cell offset code of a list entry: (dx+1) | (dy+1)<<2 | (dz+1)<<4
__host__ __device__ inline int md_code(int dx, int dy, int dz) {
  return (dx + 1) | ((dy + 1) << 2) | ((dz + 1) << 4);
}
#define MD_CODE_SELF 21  // md_code(0, 0, 0)
// Filler of the unused tail of an atom's last slab: the atom itself at a
// cell offset of +2 in every dimension (code bits 3), at least
// sqrt(3) * cell edge > rc + skin away, so a kernel that reads whole slabs
// rejects it by the cutoff test without checking the count.
#define MD_CODE_PAD 63
__host__ __device__ inline int md_pad_entry(int i) { return (int)(((unsigned)i << 6) | 63u); }
// list entry of neighbor j in the cell at offset code `code`
__host__ __device__ inline int md_make_entry(int j, int code) {
  return (int)(((unsigned)j << 6) | (unsigned)code);
}
__host__ __device__ inline int md_entry_j(unsigned e) { return (int)(e >> 6); }

// Periodic shift of a neighbour in the cell at offset d (-1, 0, +1) from
// cell c along one dimension: -prd / +prd when that cell wraps, else 0
struct Shift3 {
  double m, p;
};
__device__ __forceinline__ Shift3 shifts(int c, int nc, double prd) {
  Shift3 s;
  s.m = (c - 1 < 0) ? -prd : 0.0;
  s.p = (c + 1 >= nc) ? prd : 0.0;
  return s;
}
__device__ __forceinline__ double pick(const Shift3 &s, int d) {
  return d < 0 ? s.m : (d > 0 ? s.p : 0.0);
}

// Coordinates of the mixed form.  Each coordinate is a 32-bit fixed-point
// fraction of its periodic box edge: 2^32 units per edge, taken modulo 2^32.
// The difference of two such coordinates in 32-bit two's-complement
// arithmetic is the separation along that edge reduced to the minimum image
// (exact, with no periodic shift to decode), and one conversion turns it into
// an FP32 number of units.  A listed pair is at its minimum image whenever
// the box edge exceeds twice the list cutoff, which the mixed form requires.
// The quantisation step is prd / 2^32 (3.9e-8 sigma on the 168-sigma edge of
// a 4M-atom LJ box), below the FP32 rounding of a separation of one sigma.
__device__ __forceinline__ int md_fix(double x, double lo, double qinv) {
  return (int)(unsigned int)(unsigned long long)__double2ll_rn(__dmul_rn(x - lo, qinv));
}
__device__ __forceinline__ int4 md_xq(const double4 &p, const BoxGeom &b) {
  return make_int4(md_fix(p.x, b.lo[0], b.qinv[0]), md_fix(p.y, b.lo[1], b.qinv[1]),
                   md_fix(p.z, b.lo[2], b.qinv[2]), (int)p.w);
}
// separation a - b along one edge in fixed-point units, as an FP32 number
__device__ __forceinline__ float md_qdiff(int a, int b) {
  return (float)(int)((unsigned int)a - (unsigned int)b);
}
// u units in length units: u * (hi + lo) rounded once (the small product
// u * lo first, then one fused multiply-add; rounding u * hi first and adding
// the correction after would leave a bias of a fraction of an ulp)
__device__ __forceinline__ float md_qlen(float u, float hi, float lo) {
  return fmaf(u, hi, u * lo);
}

__host__ __device__ inline void md_entry(unsigned int e, int &j, int &dx, int &dy, int &dz) {
  j = (int)(e >> 6);
  dx = (int)(e & 3u) - 1;
  dy = (int)((e >> 2) & 3u) - 1;
  dz = (int)((e >> 4) & 3u) - 1;
}

// Slab layout of the neighbor list: entry k of atom i is at
//   nlist[((k >> 2) * stride + i) * 4 + (k & 3)]
// so that one int4 load returns four consecutive entries of an atom and the
// 32 atoms of a warp read 512 contiguous bytes per slab.
__host__ __device__ inline size_t md_slab(int k, int i, int stride) {
  return ((size_t)(k >> 2) * stride + i) * 4 + (k & 3);
}

// image flags packed as LAMMPS imageint: 10 bits per dimension, offset 512
// (src/lmptype.h IMGMAX/IMGBITS)
#define MD_IMGMAX 512
#define MD_IMGMASK 1023
__host__ __device__ inline int md_img_pack(int ix, int iy, int iz) {
  return ((iz + MD_IMGMAX) & MD_IMGMASK) << 20 | ((iy + MD_IMGMAX) & MD_IMGMASK) << 10 |
         ((ix + MD_IMGMAX) & MD_IMGMASK);
}

// 1/x in FP64: Newton's method on f(y) = 1/y - x, i.e. the iteration
// y <- y + y (1 - x y), started from the hardware reciprocal approximation
// (rcp.approx.ftz.f64) and applied twice.  For the normal, positive x used
// here the result is within two ulp of the correctly rounded quotient; the
// FP64 parity tests bound its effect on forces.
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// 1/x in FP32 from the hardware reciprocal approximation alone (one
// instruction, relative error below 2^-22); the mixed-precision kernels use it
// where the pair term's FP32 error budget is far larger.
__device__ __forceinline__ float rcp_approx_f32(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// FP64 helpers that keep a*b+c rounded twice, as the reference's x86-64
// build computes them; used wherever a comparison must be bit-exact.
__device__ __forceinline__ double dsq3(double a, double b, double c) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// The entries that one lane of an atom takes from the atom's list, G at a
// time, with the next G already loading (streaming loads).  The list holds
// each atom's entries in slabs of four: slab c of atom i is int4 number
// c * stride + i.  Several lanes per atom (TPA > 1): the atom's lanes take
// consecutive entries (lane s: entries s, s + TPA, s + 2 TPA, ...), so that
// at each gather the lanes of one atom read neighbours that sit next to each
// other in the cell-sorted order and share cache lines.  The lane's G
// offsets from its row pointer are fixed, and the pointer advances by
// TPA * G / 4 slab rows per step.  Entries past the atom's last slab read as
// `pad`.  (One lane per atom reads whole slabs and does not use this.)
template <int TPA, int G>
struct ListWalk {
  static_assert(TPA > 1 && (TPA * G) % 4 == 0, "whole slab rows per step");
  const int *p;       // row pointer of the current step
  long long off[G];   // offsets (in ints) of the lane's G entries from p
  long long adv;      // ints between steps
  int e0, ne;         // first entry of the current step; 4 x the slab count
  unsigned pad;
  unsigned cur[G], nxt[G];
  __device__ __forceinline__ ListWalk(const int *nl, int stride, int i, int nslab, int lane,
                                      unsigned pad_)
      : p(nl + (size_t)i * 4), adv((long long)(TPA * G / 4) * stride * 4), e0(lane),
        ne(nslab * 4), pad(pad_) {
#pragma unroll
    for (int u = 0; u < G; u++) {
      const int e = lane + TPA * u;
      off[u] = (long long)(e >> 2) * stride * 4 + (e & 3);
    }
    load(cur, p, e0);
  }
  __device__ __forceinline__ void load(unsigned (&v)[G], const int *q, int first) const {
#pragma unroll
    for (int u = 0; u < G; u++)
      v[u] = first + TPA * u < ne ? (unsigned)__ldcs(q + off[u]) : pad;
  }
  __device__ __forceinline__ bool more() const { return e0 < ne; }
  // start loading the next step's entries; cur holds this step's
  __device__ __forceinline__ void prefetch() { load(nxt, p + adv, e0 + TPA * G); }
  // how many of this step's entries lie before `num` (the rest are pads)
  __device__ __forceinline__ int valid(int num) const {
    return e0 >= num ? 0 : min(G, (num - e0 + TPA - 1) / TPA);
  }
  __device__ __forceinline__ void advance() {
#pragma unroll
    for (int u = 0; u < G; u++) cur[u] = nxt[u];
    p += adv;
    e0 += TPA * G;
  }
};

// Calls f(ee, m) for each group of four entries that this lane takes from
// atom i's list: ee the entries, m how many of them lie before the atom's
// count num (the rest are pads).  One lane per atom: the slabs in order, the
// next slab loading (streaming) while this one is used.  Several lanes per
// atom: ListWalk's consecutive entries.
template <int TPA, class F>
__device__ __forceinline__ void walk_list(const int *nl, int stride, int i, int num, int lane,
                                          F &&f) {
  const int nslab = (num + 3) >> 2;
  if constexpr (TPA == 1) {
    const int4 *nl4 = reinterpret_cast<const int4 *>(nl);
    int4 en = make_int4(0, 0, 0, 0);
    if (nslab > 0) en = __ldcs(&nl4[i]);
    for (int c4 = 0; c4 < nslab; c4++) {
      const int4 e4 = en;
      if (c4 + 1 < nslab) en = __ldcs(&nl4[(size_t)(c4 + 1) * stride + i]);
      const unsigned ee[4] = {(unsigned)e4.x, (unsigned)e4.y, (unsigned)e4.z, (unsigned)e4.w};
      f(ee, min(4, num - 4 * c4));
    }
  } else {
    ListWalk<TPA, 4> w(nl, stride, i, nslab, lane, (unsigned)md_pad_entry(i));
    while (w.more()) {
      w.prefetch();
      f(w.cur, w.valid(num));
      w.advance();
    }
  }
}

template <int TPA>
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
  for (int o = TPA / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int TPA>
__device__ __forceinline__ float lane_sumf(float v) {
#pragma unroll
  for (int o = TPA / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum NV doubles over the block; result valid in thread 0.  smem must hold
// NV * (blockDim.x/32) doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem) {
#pragma unroll
  for (int k = 0; k < NV; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) smem[k * nw + warp] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = 0.0;
      for (int w = 0; w < nw; w++) s += smem[k * nw + w];
      v[k] = s;
    }
  }
}

// Deterministic two-level reduction: each block writes NV partial sums, the
// last block to finish adds all partials in block order into out[0..NV-1]
// (overwrite or accumulate) and resets the counter for the next launch.
template <int NV>
__device__ __forceinline__ void block_partials_finish(double (&v)[NV], double *smem,
                                                      double *partial, unsigned int *counter,
                                                      double *out, bool accumulate) {
  block_sum<NV>(v, smem);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) partial[(size_t)blockIdx.x * NV + k] = v[k];
    __threadfence();
    unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    // every thread of the last block sums a fixed strided subset of the
    // block partials, then the block tree-reduces them: a fixed order, so
    // the result is reproducible run to run
    double s[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) s[k] = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
      for (int k = 0; k < NV; k++) s[k] += __ldcg(&partial[(size_t)b * NV + k]);
    __syncthreads();
    block_sum<NV>(s, smem);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; k++) out[k] = accumulate ? out[k] + s[k] : s[k];
      *counter = 0u;
    }
  }
}

// ---- step logic shared by the fused half-step kernel (integrate.cu) and the
// one-launch replica step (pair_lj.cu) ---------------------------------------

// Neighbor::decide (src/neighbor.cpp:1294-1309) on the device: the host
// mirrors the same schedule and reads ST_REBUILD only when the distance
// criterion decides.
__device__ __forceinline__ void md_decide_dev(int *status, int every, int delay, int check,
                                           int *dcount, volatile int *mail) {
  const int ago = status[ST_AGO] + 1;
  status[ST_AGO] = ago;
  int rebuild = 0;
  const bool candidate = ago >= delay && ago % every == 0;
  if (candidate) {
    if (!check) rebuild = 1;
    else {
      rebuild = status[ST_MOVED] != 0;
      if (rebuild && ago == (every > delay ? every : delay)) status[ST_NDANGER] += 1;
    }
  }
  bool forced = false;
  if (status[ST_FORCE_BUILD]) {  // replay after a list overflow: lists are stale
    rebuild = 1;
    forced = true;
    status[ST_FORCE_BUILD] = 0;
  }
  status[ST_MOVED] = 0;
  status[ST_REBUILD] = rebuild;
  unsigned int lo = (unsigned int)status[ST_STEP_LO] + 1u;
  if (lo == 0u) status[ST_STEP_HI] += 1;
  status[ST_STEP_LO] = (int)lo;
  if (check && candidate && !forced) {
    // a decision the host waits for (the distance criterion): the flag
    // first, then, after a system-wide fence, the new decision count
    const int k = *dcount + 1;
    *dcount = k;
    mail[0] = rebuild;
    __threadfence_system();
    mail[1] = k;
  }
}

__device__ __forceinline__ void md_record_row_dev(int *status, const double *ev, double *rows,
                                               int cap) {
  const int r = status[ST_ROW];
  if (r < cap) {
    double *row = rows + 9 * (size_t)r;
    const long long step = ((long long)(unsigned int)status[ST_STEP_HI] << 32) |
                           (long long)(unsigned int)status[ST_STEP_LO];
    row[0] = (double)step;
    row[1] = ev[7];
    row[2] = ev[0];
    for (int k = 0; k < 6; k++) row[3 + k] = ev[1 + k];
  }
  status[ST_ROW] = r + 1;
}

// FixNVE::final_integrate of this step for sorted atom i with its force
// (fx, fy, fz), the kinetic-energy term of the thermo output (KE, into ke),
// then FixNVE::initial_integrate of the next step (src/fix_nve.cpp:65-142):
// every product and sum rounded separately as in the reference.  The new
// position goes to x4_out (x4_in itself for an update in place) and, in the
// mixed form, its fixed-point copy to xq_out.  Returns whether the atom moved
// more than half the skin since the last build (xhold, check yes).
template <bool KE>
__device__ __forceinline__ bool md_nve_step_atom(int i, int stride, double dtv, double dtf,
                                                 const double *__restrict__ mass,
                                                 const double4 *x4_in, double4 *x4_out,
                                                 double *__restrict__ v, double fx, double fy,
                                                 double fz, int4 *__restrict__ xq_out,
                                                 const BoxGeom &box,
                                                 const double4 *__restrict__ xhold,
                                                 double triggersq, double &ke) {
  double4 p = x4_in[i];
  const double m = mass[(int)p.w];
  const double dtfm = dtf / m;
  double vx = __dadd_rn(v[i], __dmul_rn(dtfm, fx));
  double vy = __dadd_rn(v[stride + i], __dmul_rn(dtfm, fy));
  double vz = __dadd_rn(v[2 * stride + i], __dmul_rn(dtfm, fz));
  // ComputeTemp::compute_scalar term of this step (src/compute_temp.cpp:84-86)
  if (KE) ke = (vx * vx + vy * vy + vz * vz) * m;
  vx = __dadd_rn(vx, __dmul_rn(dtfm, fx));
  vy = __dadd_rn(vy, __dmul_rn(dtfm, fy));
  vz = __dadd_rn(vz, __dmul_rn(dtfm, fz));
  p.x = __dadd_rn(p.x, __dmul_rn(dtv, vx));
  p.y = __dadd_rn(p.y, __dmul_rn(dtv, vy));
  p.z = __dadd_rn(p.z, __dmul_rn(dtv, vz));
  v[i] = vx;
  v[stride + i] = vy;
  v[2 * stride + i] = vz;
  x4_out[i] = p;
  if (xq_out) xq_out[i] = md_xq(p, box);
  if (xhold) {
    const double4 h = xhold[i];
    const double rsq = dsq3(__dsub_rn(p.x, h.x), __dsub_rn(p.y, h.y), __dsub_rn(p.z, h.z));
    return rsq > triggersq;
  }
  return false;
}

// The same step for atom i with its force read from f and its position
// updated in place (k_nve_fused, the replica step).
template <bool KE>
__device__ __forceinline__ bool md_nve_fused_atom(int i, int stride, double dtv, double dtf,
                                                  const double *__restrict__ mass,
                                                  double4 *__restrict__ x4, double *__restrict__ v,
                                                  const double *__restrict__ f,
                                                  int4 *__restrict__ xq, const BoxGeom &box,
                                                  const double4 *__restrict__ xhold,
                                                  double triggersq, double &ke) {
  return md_nve_step_atom<KE>(i, stride, dtv, dtf, mass, x4, x4, v, f[i], f[stride + i],
                              f[2 * stride + i], xq, box, xhold, triggersq, ke);
}

// ---- one-launch MD steps (k_lj_step, k_eam_force with STEP) ---------------
// A force kernel that also advances the atoms: after its pair loop each
// atom's first lane applies this step's final half-step and the next step's
// initial half-step.  The neighbour gathers read the positions in `cur`; the
// new positions go to `nxt`, a second buffer, so no update can reach a gather
// of the same launch; the host swaps the two buffers after the launch.  Mixed
// form: cur/nxt are the fixed-point coordinates and the FP64 positions x4
// are updated in place (the mixed gathers never read them); FP64 form:
// cur/nxt are the FP64 positions.
struct StepArgs {
  double dtv, dtf, triggersq;
  const double *mass;
  double4 *x4;      // mixed form: FP64 positions, updated in place
  const void *cur;  // positions the gathers read: int4 (mixed) or double4
  void *nxt;        // positions after the next initial half-step
  double *v;
  const double4 *xhold;
  int *status, *dcount, *mail;
  double *rows;
  int rows_cap, every, delay, check;
};

// The atom's half-steps, by its first lane, with its summed force.  The
// forces stay in registers on an ordinary step: within a run chunk nothing
// reads them (a chunk's last step is the two-kernel form, which stores them
// for the next chunk's first half-step and for downloads); an output step
// stores them all the same.
template <bool OUT, bool MIXED>
__device__ __forceinline__ bool md_step_atom(const StepArgs &s, int i, int stride, double *f,
                                             double fx, double fy, double fz,
                                             const BoxGeom &box, double &ke) {
  if (OUT) {
    f[i] = fx;
    f[stride + i] = fy;
    f[2 * stride + i] = fz;
  }
  if (MIXED)
    return md_nve_step_atom<OUT>(i, stride, s.dtv, s.dtf, s.mass, s.x4, s.x4, s.v, fx, fy, fz,
                                 static_cast<int4 *>(s.nxt), box, s.xhold, s.triggersq, ke);
  return md_nve_step_atom<OUT>(i, stride, s.dtv, s.dtf, s.mass,
                               static_cast<const double4 *>(s.cur),
                               static_cast<double4 *>(s.nxt), s.v, fx, fy, fz, nullptr, box,
                               s.xhold, s.triggersq, ke);
}

// The end of a one-launch step (every thread of the block).  The
// displacement flag goes to the status word.  On an output step the last
// block to finish adds the energy and virial (ev[0..6]: written, or added to
// what an earlier pass of the step left there) and the kinetic energy
// (ev[7]) in block order, records the thermo row and makes the next step's
// rebuild decision, as k_nve_fused does.  Other steps end with no
// block-completion count: one returning atomic per block lengthens every
// block's life (with that count on every step the 4M-atom LJ step ran at
// 5,020 Matom-steps/s, without it at 5,723), so their decision is a
// one-thread kernel launched after the step kernel.  red: 8 x (warps per
// block) doubles of shared memory.
template <bool OUT>
__device__ __forceinline__ void md_step_tail(const StepArgs &s, bool moved, const double (&acc)[7],
                                             double ke, double *red, double *partial,
                                             unsigned int *counter, double *ev,
                                             bool accumulate) {
  if (s.xhold && __any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) {
    atomicOr(&s.status[ST_MOVED], 1);
    if (OUT) __threadfence();  // the flag is visible before this block counts itself done
  }
  if (!OUT) return;
  __shared__ bool last;
  double v8[8];
#pragma unroll
  for (int k = 0; k < 7; k++) v8[k] = acc[k];
  v8[7] = ke;
  block_sum<8>(v8, red);
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 8; k++) partial[(size_t)blockIdx.x * 8 + k] = v8[k];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // block partials added in a fixed order: reproducible run to run
  double sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < 8; k++) sum[k] += __ldcg(&partial[(size_t)b * 8 + k]);
  __syncthreads();
  block_sum<8>(sum, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 7; k++) ev[k] = accumulate ? ev[k] + sum[k] : sum[k];
    ev[7] = sum[7];
    md_record_row_dev(s.status, ev, s.rows, s.rows_cap);
    md_decide_dev(s.status, s.every, s.delay, s.check, s.dcount, s.mail);
    *counter = 0u;
  }
}
