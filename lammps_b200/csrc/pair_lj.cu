// pair_lj.cu -- pair_style lj/cut force kernels over the full neighbor list.
//
// Replaces PairLJCut::compute (src/pair_lj_cut.cpp:68-141).  With a full
// list each atom sums its own force, so no atomics, no ghost forces and no
// reverse communication are needed; energy and virial are accumulated as
// half of every pair term (the reference's ev_tally with newton on gives the
// same totals, src/pair.cpp:769-855) and reduced deterministically.
//
// FP64 form: arithmetic identical to the reference per pair; the periodic
// image is x_j + s*L and rsq is rounded after every operation, so the
// rsq < cutsq decision is the reference's.
// Mixed form: positions are read as 32-bit fixed-point fractions of the box
// edge (md_xq, int4, 16 B per gather); a separation is one integer
// subtraction and one conversion per component, already at the minimum
// image; the pair force is FP32 and each atom's force, energy and virial are
// summed in FP64.
//
// Memory-level parallelism: each thread reads four list entries with one
// 16-byte load (slab layout, md_slab).  The FP64 kernel issues a slab's four
// neighbor gathers before using any of them and forms 1/rsq by Newton's
// method from the hardware reciprocal (rcp_nr); for an atom away from the
// box faces it skips the periodic-shift decode.  The mixed kernel works on
// four slabs at a time with the next four already loading, evaluates every
// entry branch-free with the one-instruction FP32 reciprocal, and adds the
// FP32 force sum of each eight entries to the FP64 accumulator.
#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "md_state.h"

namespace {

struct PairArgs {
  int n, stride, ntp1;
  BoxGeom box;
  Reps reps;  // replica boxes of a batched context
  const double *tables;
  const int *cell, *nlist, *numneigh, *orig;
  double *f;
  double *partial;
  unsigned int *counter;
  double *ev;
  double *eatom, *vatom;
};

__device__ __forceinline__ void decode(unsigned int e, int &j, int &dx, int &dy, int &dz) {
  md_entry(e, j, dx, dy, dz);
}

// lane sums of one atom's force (and per-atom energy/virial), stored by lane 0
template <int TPA, bool EV, bool ATOM>
__device__ __forceinline__ void lj_atom_store(const PairArgs &a, int i, int lane, bool active,
                                              double fx, double fy, double fz,
                                              const double (&acc)[7]) {
  fx = lane_sum<TPA>(fx);
  fy = lane_sum<TPA>(fy);
  fz = lane_sum<TPA>(fz);
  if (active && lane == 0) {
    a.f[i] = fx;
    a.f[a.stride + i] = fy;
    a.f[2 * a.stride + i] = fz;
  }
  if (EV && ATOM) {
    double e[7];
#pragma unroll
    for (int k = 0; k < 7; k++) e[k] = lane_sum<TPA>(acc[k]);
    if (active && lane == 0) {
      const int o = a.orig[i];
      if (a.eatom) a.eatom[o] = e[0];
      if (a.vatom)
#pragma unroll
        for (int k = 0; k < 6; k++) a.vatom[6 * (size_t)o + k] = e[1 + k];
    }
  }
}

// One atom's pair forces in FP64 (this thread's lane of the TPA threads of
// atom i): adds to fx, fy, fz (and to acc with EV).  `tab` is the per-type
// table in shared memory (unused with SINGLE).
template <int TPA, bool EV, bool SINGLE, bool BATCH>
__device__ __forceinline__ void lj_atom_fp64(const PairArgs &a, const double4 *__restrict__ x4,
                                             const double *tab, int nt2, int i, int lane,
                                             bool active, double &fx, double &fy, double &fz,
                                             double (&acc)[7]) {
  if (active) {
    double cutsq1 = 0, lj1 = 0, lj2 = 0, lj3 = 0, lj4 = 0, off = 0;
    if (SINGLE) {
      const int k11 = a.ntp1 + 1;
      cutsq1 = __ldg(&a.tables[TAB_CUTSQ * TABSZ + k11]);
      lj1 = __ldg(&a.tables[TAB_LJ1 * TABSZ + k11]);
      lj2 = __ldg(&a.tables[TAB_LJ2 * TABSZ + k11]);
      lj3 = __ldg(&a.tables[TAB_LJ3 * TABSZ + k11]);
      lj4 = __ldg(&a.tables[TAB_LJ4 * TABSZ + k11]);
      off = __ldg(&a.tables[TAB_OFFSET * TABSZ + k11]);
    }
    const double4 xi = x4[i];
    const int ti = (int)xi.w;
    int cx, cy, cz;
    md_cell_unpack(a.cell[i], cx, cy, cz);
    const BoxGeom &box = BATCH ? a.reps.box[a.reps.rep_of_atom[i]] : a.box;
    const Shift3 sx = shifts(cx, box.ncell[0], box.prd[0]);
    const Shift3 sy = shifts(cy, box.ncell[1], box.prd[1]);
    const Shift3 sz = shifts(cz, box.ncell[2], box.prd[2]);
    const int num = a.numneigh[i];
    const int4 *nl4 = reinterpret_cast<const int4 *>(a.nlist);
    // An atom whose 27 neighbour cells all lie inside the box has no
    // periodic image among its neighbours: x_j + 0.0 is x_j exactly, so the
    // offset decode and the shift are skipped (same results bit for bit).
    const bool interior = cx >= 1 && cx + 2 <= box.ncell[0] && cy >= 1 &&
                          cy + 2 <= box.ncell[1] && cz >= 1 && cz + 2 <= box.ncell[2];
    const int nslab = (num + 3) >> 2;
    auto slabs = [&](auto wrap_tag) {
    constexpr bool WRAP = decltype(wrap_tag)::value;
    // four entries ee, of which the first m lie before the atom's count
    auto four = [&](const unsigned (&ee)[4], int m) {
      double4 xj[4];
#pragma unroll
      for (int u = 0; u < 4; u++) xj[u] = x4[u < m ? md_entry_j(ee[u]) : i];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (u >= m) break;
        double delx, dely, delz;
        if (WRAP) {
          int j, dx, dy, dz;
          decode(ee[u], j, dx, dy, dz);
          delx = __dsub_rn(xi.x, __dadd_rn(xj[u].x, pick(sx, dx)));
          dely = __dsub_rn(xi.y, __dadd_rn(xj[u].y, pick(sy, dy)));
          delz = __dsub_rn(xi.z, __dadd_rn(xj[u].z, pick(sz, dz)));
        } else {
          delx = __dsub_rn(xi.x, xj[u].x);
          dely = __dsub_rn(xi.y, xj[u].y);
          delz = __dsub_rn(xi.z, xj[u].z);
        }
        const double rsq = dsq3(delx, dely, delz);
        const int tt = ti * a.ntp1 + (int)xj[u].w;
        const double cs = SINGLE ? cutsq1 : tab[0 * nt2 + tt];
        if (rsq < cs) {
          const double c1 = SINGLE ? lj1 : tab[1 * nt2 + tt];
          const double c2 = SINGLE ? lj2 : tab[2 * nt2 + tt];
          const double r2inv = rcp_nr(rsq);
          const double r6inv = r2inv * r2inv * r2inv;
          const double forcelj = r6inv * (c1 * r6inv - c2);
          const double fpair = forcelj * r2inv;
          fx += delx * fpair;
          fy += dely * fpair;
          fz += delz * fpair;
          if (EV) {
            const double c3 = SINGLE ? lj3 : tab[3 * nt2 + tt];
            const double c4 = SINGLE ? lj4 : tab[4 * nt2 + tt];
            const double co = SINGLE ? off : tab[5 * nt2 + tt];
            const double evdwl = r6inv * (c3 * r6inv - c4) - co;
            acc[0] += 0.5 * evdwl;
            const double hf = 0.5 * fpair;
            acc[1] += delx * delx * hf;
            acc[2] += dely * dely * hf;
            acc[3] += delz * delz * hf;
            acc[4] += delx * dely * hf;
            acc[5] += delx * delz * hf;
            acc[6] += dely * delz * hf;
          }
        }
      }
    };
    if constexpr (TPA == 1) {
      // the next slab's entries load (streaming) while this slab is used
      int4 en = make_int4(0, 0, 0, 0);
      if (nslab > 0) en = __ldcs(&nl4[i]);
      for (int c4 = 0; c4 < nslab; c4++) {
        const int4 e4 = en;
        if (c4 + 1 < nslab) en = __ldcs(&nl4[(size_t)(c4 + 1) * a.stride + i]);
        const unsigned int ee[4] = {(unsigned int)e4.x, (unsigned int)e4.y, (unsigned int)e4.z,
                                    (unsigned int)e4.w};
        four(ee, min(4, num - 4 * c4));
      }
    } else {
      // the atom's lanes take consecutive entries (ListWalk)
      ListWalk<TPA, 4> w(a.nlist, a.stride, i, nslab, lane, (unsigned)md_pad_entry(i));
      while (w.more()) {
        w.prefetch();
        four(w.cur, w.valid(num));
        w.advance();
      }
    }
    };
    if (interior) slabs(std::false_type{});
    else slabs(std::true_type{});
  }
}

// One atom's pair forces in the mixed form (FP32 pair math, FP64 sums), as
// lj_atom_fp64.  `tabf` is the per-type table in shared memory.  Separations
// come from the fixed-point coordinates (md_xq): per component one 32-bit
// subtraction and one conversion give the minimum-image separation in units
// of prd/2^32, so no periodic offset is decoded.
//   ISO (equal box edges: one unit in every dimension): the pair arithmetic
//   runs on separations in units; 1/r^2 is brought to length units by the
//   FP32 pair hi + lo of 1/unit^2 (md_qlen), and an FP32 force sum (units x
//   force/length) is scaled by the exact FP64 unit length as it joins the
//   FP64 accumulator.
//   Otherwise each component is scaled to length units first (md_qlen).
// The scale constants are never a single rounded FP32 value, which would
// bias every pair term the same way.
// A pad entry names the atom itself (zero separation), which the r^2 > 0
// test rejects.
// One thread per atom (TPA 1): the thread walks its list four slabs (16
// entries) at a time.  Several threads per atom: the atom's lanes take
// consecutive entries (lane s: entries s, s + TPA, s + 2 TPA, ...), so that
// at each gather the lanes of one atom read neighbours that sit next to each
// other in the cell-sorted order and share cache lines; each lane then loads
// one 4-byte entry per gather instead of a 16-byte slab per four.
template <int TPA, bool EV, bool SINGLE, bool BATCH, bool ISO>
__device__ __forceinline__ void lj_atom_mixed(const PairArgs &a, const int4 *__restrict__ xq,
                                              const float *tabf, int nt2, int i, int lane,
                                              bool active, double &fx, double &fy, double &fz,
                                              double (&acc)[7]) {
  if (!active) return;
  const BoxGeom &box = BATCH ? a.reps.box[a.reps.rep_of_atom[i]] : a.box;
  const float qx = box.qs[0], qy = box.qs[1], qz = box.qs[2];
  const float qxl = box.qs_lo[0], qyl = box.qs_lo[1], qzl = box.qs_lo[2];
  // ISO: 1/r^2 in units times (q2h + q2l) is 1/r^2 in length units, and a
  // force sum in units times qd (exact) is the force
  const float q2h = box.q2inv, q2l = box.q2inv_lo;
  const double qd = box.prd[0] * (1.0 / 4294967296.0);
  float cutsq1 = 0, lj1 = 0, lj2 = 0, lj3 = 0, lj4 = 0, off = 0;
  if (SINGLE) {
    const int k11 = a.ntp1 + 1;
    const double cs = __ldg(&a.tables[TAB_CUTSQ * TABSZ + k11]);
    cutsq1 = ISO ? (float)(cs / (qd * qd)) : (float)cs;
    lj1 = (float)__ldg(&a.tables[TAB_LJ1 * TABSZ + k11]);
    lj2 = (float)__ldg(&a.tables[TAB_LJ2 * TABSZ + k11]);
    lj3 = (float)__ldg(&a.tables[TAB_LJ3 * TABSZ + k11]);
    lj4 = (float)__ldg(&a.tables[TAB_LJ4 * TABSZ + k11]);
    off = (float)__ldg(&a.tables[TAB_OFFSET * TABSZ + k11]);
  }
  const int4 xi = xq[i];
  const int ti = xi.w;
  const int nslab = (a.numneigh[i] + 3) >> 2;
  const int pe = md_pad_entry(i);
  // The pair forces of N gathered neighbours, summed in FP32; the group sum
  // (and, with EV, the group's energy and virial sums) joins the atom's FP64
  // accumulators.
  auto group = [&](const int4 *xj, auto n_c) {
    constexpr int N = decltype(n_c)::value;
    float cfx = 0.f, cfy = 0.f, cfz = 0.f;
    float ce[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // EV: this group's FP32 sums
#pragma unroll
    for (int u = 0; u < N; u++) {
      // x_i - x_j at the minimum image, in units (ISO) or lengths
      float delx = md_qdiff(xi.x, xj[u].x);
      float dely = md_qdiff(xi.y, xj[u].y);
      float delz = md_qdiff(xi.z, xj[u].z);
      if (!ISO) {
        delx = md_qlen(delx, qx, qxl);
        dely = md_qlen(dely, qy, qyl);
        delz = md_qlen(delz, qz, qzl);
      }
      const float rsq = delx * delx + dely * dely + delz * delz;
      const int tt = ti * a.ntp1 + xj[u].w;
      // (the cutoff in units only selects pairs: its rounding biases no term)
      const float cs = SINGLE ? cutsq1 : (ISO ? tabf[0 * nt2 + tt] * q2h : tabf[0 * nt2 + tt]);
      const float c1 = SINGLE ? lj1 : tabf[1 * nt2 + tt];
      const float c2 = SINGLE ? lj2 : tabf[2 * nt2 + tt];
      const bool in = rsq < cs && rsq > 0.f;
      const float r2inv = ISO ? md_qlen(rcp_approx_f32(rsq), q2h, q2l) : rcp_approx_f32(rsq);
      const float r6inv = r2inv * r2inv * r2inv;
      const float fpair = in ? r6inv * (c1 * r6inv - c2) * r2inv : 0.f;
      cfx = fmaf(delx, fpair, cfx);
      cfy = fmaf(dely, fpair, cfy);
      cfz = fmaf(delz, fpair, cfz);
      if (EV) {
        const float c3 = SINGLE ? lj3 : tabf[3 * nt2 + tt];
        const float c4 = SINGLE ? lj4 : tabf[4 * nt2 + tt];
        const float co = SINGLE ? off : tabf[5 * nt2 + tt];
        const float evdwl = in ? r6inv * (c3 * r6inv - c4) - co : 0.f;
        ce[0] = fmaf(0.5f, evdwl, ce[0]);
        // the virial wants separations in length units
        const float lx = ISO ? md_qlen(delx, qx, qxl) : delx,
                    ly = ISO ? md_qlen(dely, qx, qxl) : dely,
                    lz = ISO ? md_qlen(delz, qx, qxl) : delz;
        const float hf = 0.5f * fpair;
        ce[1] = fmaf(lx * lx, hf, ce[1]);
        ce[2] = fmaf(ly * ly, hf, ce[2]);
        ce[3] = fmaf(lz * lz, hf, ce[3]);
        ce[4] = fmaf(lx * ly, hf, ce[4]);
        ce[5] = fmaf(lx * lz, hf, ce[5]);
        ce[6] = fmaf(ly * lz, hf, ce[6]);
      }
    }
    // the energy and virial terms join the FP64 sums once per group, as the
    // forces do
    if (EV)
#pragma unroll
      for (int k = 0; k < 7; k++) acc[k] += (double)ce[k];
    if (ISO) {
      fx = fma((double)cfx, qd, fx);
      fy = fma((double)cfy, qd, fy);
      fz = fma((double)cfz, qd, fz);
    } else {
      fx += (double)cfx;
      fy += (double)cfy;
      fz += (double)cfz;
    }
  };
  if constexpr (TPA == 1) {
    // Four slabs (16 entries) per iteration: the sixteen gathers are in
    // flight together, and the next four slabs' entries are loaded
    // (streaming, evict-first) before these are used, so the list's DRAM
    // latency overlaps the gathers and the arithmetic of the slabs before
    // them.  Slabs past the atom's count, and the tail of its last slab, hold
    // pad entries, which the r^2 > 0 test rejects, so no per-entry count
    // check is needed.  The forces of each eight entries are summed in FP32.
    const int4 *nl4 = reinterpret_cast<const int4 *>(a.nlist);
    const int4 pad4 = make_int4(pe, pe, pe, pe);
    auto slab = [&](int c) { return c < nslab ? __ldcs(&nl4[(size_t)c * a.stride + i]) : pad4; };
    int c4 = 0;
    int4 a0 = slab(0), a1 = slab(1), a2 = slab(2), a3 = slab(3);
    while (c4 < nslab) {
      const int cn = c4 + 4;
      const int4 b0 = slab(cn), b1 = slab(cn + 1), b2 = slab(cn + 2), b3 = slab(cn + 3);
      const unsigned int eall[16] = {(unsigned)a0.x, (unsigned)a0.y, (unsigned)a0.z, (unsigned)a0.w,
                                     (unsigned)a1.x, (unsigned)a1.y, (unsigned)a1.z, (unsigned)a1.w,
                                     (unsigned)a2.x, (unsigned)a2.y, (unsigned)a2.z, (unsigned)a2.w,
                                     (unsigned)a3.x, (unsigned)a3.y, (unsigned)a3.z, (unsigned)a3.w};
      int4 xall[16];
#pragma unroll
      for (int u = 0; u < 16; u++) xall[u] = __ldg(&xq[md_entry_j(eall[u])]);
      group(xall, std::integral_constant<int, 8>{});
      group(xall + 8, std::integral_constant<int, 8>{});
      a0 = b0;
      a1 = b1;
      a2 = b2;
      a3 = b3;
      c4 = cn;
    }
  } else {
    // G entries per lane per iteration (their gathers in flight together),
    // the next G entries already loading; entries past the last slab are
    // pads.  The forces of each lane's G entries are summed in FP32.
    constexpr int G = TPA == 2 ? 8 : 4;
    ListWalk<TPA, G> w(a.nlist, a.stride, i, nslab, lane, (unsigned)pe);
    while (w.more()) {
      w.prefetch();
      int4 xall[G];
#pragma unroll
      for (int u = 0; u < G; u++) xall[u] = __ldg(&xq[md_entry_j(w.cur[u])]);
      group(xall, std::integral_constant<int, G>{});
      w.advance();
    }
  }
}

template <int TPA, bool EV, bool ATOM, bool SINGLE, bool BATCH>
__global__ void __launch_bounds__(128) k_lj_fp64(PairArgs a, const double4 *__restrict__ x4) {
  __shared__ double tab[6 * TABSZ];
  __shared__ double red[7 * 4];
  const int nt2 = a.ntp1 * a.ntp1;
  if (!SINGLE) {
    for (int k = threadIdx.x; k < 6 * nt2; k += blockDim.x)
      tab[k] = a.tables[(TAB_CUTSQ + k / nt2) * TABSZ + k % nt2];
    __syncthreads();
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / TPA, lane = t % TPA;
  const bool active = i < a.n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  lj_atom_fp64<TPA, EV, SINGLE, BATCH>(a, x4, tab, nt2, i, lane, active, fx, fy, fz, acc);
  lj_atom_store<TPA, EV, ATOM>(a, i, lane, active, fx, fy, fz, acc);
  if (EV) block_partials_finish<7>(acc, red, a.partial, a.counter, a.ev, false);
}

template <int TPA, bool EV, bool ATOM, bool SINGLE, bool BATCH, bool ISO>
__global__ void __launch_bounds__(128) k_lj_mixed(PairArgs a, const int4 *__restrict__ xq) {
  __shared__ float tabf[6 * TABSZ];
  __shared__ double red[7 * 4];
  const int nt2 = a.ntp1 * a.ntp1;
  if (!SINGLE) {
    for (int k = threadIdx.x; k < 6 * nt2; k += blockDim.x)
      tabf[k] = (float)a.tables[(TAB_CUTSQ + k / nt2) * TABSZ + k % nt2];
    __syncthreads();
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / TPA, lane = t % TPA;
  const bool active = i < a.n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  lj_atom_mixed<TPA, EV, SINGLE, BATCH, ISO>(a, xq, tabf, nt2, i, lane, active, fx, fy, fz, acc);
  lj_atom_store<TPA, EV, ATOM>(a, i, lane, active, fx, fy, fz, acc);
  if (EV) block_partials_finish<7>(acc, red, a.partial, a.counter, a.ev, false);
}

// One MD step of lj/cut after the neighbor list, in one launch: each atom's
// pair forces (lj_atom_mixed / lj_atom_fp64, the same code and order as
// k_lj_mixed / k_lj_fp64), then, by the atom's first lane, the final
// half-step of this step, its kinetic-energy term on an output step and the
// initial half-step of the next (md_step_atom, the arithmetic of
// k_nve_fused), with the position buffers and the step's end described at
// StepArgs and md_step_tail.
template <int TPA, bool OUT, bool SINGLE, bool MIXED>
__global__ void __launch_bounds__(128) k_lj_step(PairArgs a, StepArgs s) {
  __shared__ double tab[6 * TABSZ];
  __shared__ double red[8 * 4];
  float *tabf = reinterpret_cast<float *>(tab);
  const int nt2 = a.ntp1 * a.ntp1;
  if (!SINGLE) {
    for (int k = threadIdx.x; k < 6 * nt2; k += blockDim.x) {
      const double t = a.tables[(TAB_CUTSQ + k / nt2) * TABSZ + k % nt2];
      if (MIXED) tabf[k] = (float)t;
      else tab[k] = t;
    }
    __syncthreads();
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / TPA, lane = t % TPA;
  const bool active = i < a.n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (MIXED)
    lj_atom_mixed<TPA, OUT, SINGLE, false, true>(a, static_cast<const int4 *>(s.cur), tabf, nt2,
                                                  i, lane, active, fx, fy, fz, acc);
  else
    lj_atom_fp64<TPA, OUT, SINGLE, false>(a, static_cast<const double4 *>(s.cur), tab, nt2, i,
                                          lane, active, fx, fy, fz, acc);
  fx = lane_sum<TPA>(fx);
  fy = lane_sum<TPA>(fy);
  fz = lane_sum<TPA>(fz);
  double ke = 0.0;
  bool moved = false;
  if (active && lane == 0)
    moved = md_step_atom<OUT, MIXED>(s, i, a.stride, a.f, fx, fy, fz, a.box, ke);
  md_step_tail<OUT>(s, moved, acc, ke, red, a.partial, a.counter, a.ev, false);
}

// One MD step of every replica of a batched context in one launch.  Cluster g
// (rep_cs CTAs) owns a fixed set of whole replicas: the concatenation of the
// atom ranges ranges[first[g] .. first[g+1]).  Each CTA takes an equal share
// of that concatenation.  A replica's atoms interact only with each other, so
// the step needs no grid-wide ordering:
//   1. pair forces of the share's atoms (lj_atom_*, the same code and order as
//      k_lj_fp64 / k_lj_mixed);
//   2. a cluster barrier: every position of the group has been read;
//   3. FixNVE final half-step of this step and initial half-step of the next
//      for the share's atoms (md_nve_fused_atom, as k_nve_fused);
//   4. the last CTA of the grid to finish makes the next step's rebuild
//      decision, with every CTA's displacement flag (as k_nve_fused).
// The per-atom arithmetic is the graph path's, so both give the same bits.
struct RepStepArgs {
  const int *first;   // per group: first range, ngroups + 1 entries
  const int2 *ranges; // (start, count) of sorted atoms
  double dtv, dtf, triggersq;
  const double *mass;
  double4 *x4;
  double *v;
  const double4 *xhold;
  int *status, *dcount, *mail;
  unsigned int *counter;
  int every, delay, check;
};

// sorted atom index of position k in the concatenation of ranges [r0, r1)
__device__ __forceinline__ int rep_atom(const int2 *__restrict__ ranges, int r0, int r1, int k) {
  for (int r = r0; r < r1; r++) {
    const int2 rg = ranges[r];
    if (k < rg.y) return rg.x + k;
    k -= rg.y;
  }
  return -1;
}

template <int TPA, bool MIXED, bool SINGLE, bool ISO>
__global__ void __launch_bounds__(512) k_rep_step(PairArgs a, const double4 *__restrict__ x4,
                                                   const int4 *__restrict__ xq, RepStepArgs s) {
  namespace cg = cooperative_groups;
  __shared__ double tab[6 * TABSZ];
  __shared__ bool last;
  const int nt2 = a.ntp1 * a.ntp1;
  if (!SINGLE) {
    for (int k = threadIdx.x; k < 6 * nt2; k += blockDim.x)
      tab[k] = a.tables[(TAB_CUTSQ + k / nt2) * TABSZ + k % nt2];
  }
  float *tabf = reinterpret_cast<float *>(tab);
  if (!SINGLE && MIXED) {
    __syncthreads();
    for (int k = threadIdx.x; k < 6 * nt2; k += blockDim.x) tabf[k] = (float)tab[k];
  }
  __syncthreads();
  cg::cluster_group cl = cg::this_cluster();
  const int cs = (int)cl.num_blocks(), cr = (int)cl.block_rank();
  const int g = blockIdx.x / cs;
  const int r0 = s.first[g], r1 = s.first[g + 1];
  int total = 0;
  for (int r = r0; r < r1; r++) total += s.ranges[r].y;
  const int k0 = (int)((long long)total * cr / cs), k1 = (int)((long long)total * (cr + 1) / cs);
  // 1. forces: TPA threads per atom, every thread takes the same trip count
  const int work = (k1 - k0) * TPA;
  for (int base = 0; base < work; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const int lane = t % TPA;
    const bool active = t < work;
    const int i = active ? rep_atom(s.ranges, r0, r1, k0 + t / TPA) : 0;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (MIXED)
      lj_atom_mixed<TPA, false, SINGLE, true, ISO>(a, xq, tabf, nt2, i, lane, active, fx, fy, fz,
                                                   acc);
    else
      lj_atom_fp64<TPA, false, SINGLE, true>(a, x4, tab, nt2, i, lane, active, fx, fy, fz, acc);
    lj_atom_store<TPA, false, false>(a, i, lane, active, fx, fy, fz, acc);
  }
  // 2. every CTA of the cluster has read the group's positions
  cl.sync();
  // 3. half-steps of the share's atoms
  bool moved = false;
  for (int k = k0 + (int)threadIdx.x; k < k1; k += blockDim.x) {
    const int i = rep_atom(s.ranges, r0, r1, k);
    double ke = 0.0;
    moved |= md_nve_fused_atom<false>(i, a.stride, s.dtv, s.dtf, s.mass, const_cast<double4 *>(x4),
                                      s.v, a.f, MIXED ? const_cast<int4 *>(xq) : nullptr,
                                      a.reps.box[a.reps.rep_of_atom[i]], s.xhold, s.triggersq, ke);
  }
  if (s.xhold && __any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) {
    atomicExch(&s.status[ST_MOVED], 1);
    __threadfence();  // the flag is visible before this block counts itself done
  }
  // 4. the last CTA to finish makes the next step's rebuild decision
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(s.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    md_decide_dev(s.status, s.every, s.delay, s.check, s.dcount, s.mail);
    *s.counter = 0u;
  }
}

template <int TPA, bool MIXED, bool ISO>
cudaError_t launch_rep_t(b200_ctx *c, const PairArgs &a, const RepStepArgs &s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(c->rep_groups * c->rep_cs), 1, 1);
  cfg.blockDim = dim3((unsigned)c->rep_block, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)c->rep_cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (c->ntypes == 1)
    return cudaLaunchKernelEx(&cfg, k_rep_step<TPA, MIXED, true, ISO>, a, (const double4 *)c->x4,
                              (const int4 *)c->xq, s);
  return cudaLaunchKernelEx(&cfg, k_rep_step<TPA, MIXED, false, ISO>, a, (const double4 *)c->x4,
                            (const int4 *)c->xq, s);
}

template <int TPA, bool EV, bool ATOM, bool SINGLE, bool BATCH>
void launch_t(b200_ctx *c, const PairArgs &a) {
  const int B = 128;
  const int grid = md_blocks((long long)a.n * TPA, B);
  if (c->prec == B200_PREC_MIXED && md_q_iso(c))
    k_lj_mixed<TPA, EV, ATOM, SINGLE, BATCH, true><<<grid, B, 0, c->stream>>>(a, c->xq);
  else if (c->prec == B200_PREC_MIXED)
    k_lj_mixed<TPA, EV, ATOM, SINGLE, BATCH, false><<<grid, B, 0, c->stream>>>(a, c->xq);
  else
    k_lj_fp64<TPA, EV, ATOM, SINGLE, BATCH><<<grid, B, 0, c->stream>>>(a, c->x4);
  c->launches++;
}

template <int TPA, bool BATCH>
void launch_tb(b200_ctx *c, const PairArgs &a, bool ev, bool atom, bool single) {
  if (!ev) {
    if (single) launch_t<TPA, false, false, true, BATCH>(c, a);
    else launch_t<TPA, false, false, false, BATCH>(c, a);
  } else if (!atom) {
    if (single) launch_t<TPA, true, false, true, BATCH>(c, a);
    else launch_t<TPA, true, false, false, BATCH>(c, a);
  } else {
    if (single) launch_t<TPA, true, true, true, BATCH>(c, a);
    else launch_t<TPA, true, true, false, BATCH>(c, a);
  }
}

template <int TPA>
void launch_tpa(b200_ctx *c, const PairArgs &a, bool ev, bool atom, bool single) {
  if (c->nrep) launch_tb<TPA, true>(c, a, ev, atom, single);
  else launch_tb<TPA, false>(c, a, ev, atom, single);
}

}  // namespace

static PairArgs pair_args(b200_ctx *c, double *eatom, double *vatom) {
  PairArgs a;
  a.n = c->n;
  a.stride = c->stride;
  a.ntp1 = c->ntypes + 1;
  a.box = c->box;
  a.reps = c->reps();
  a.tables = c->tables_dev;
  a.cell = c->cell;
  a.nlist = c->nlist;
  a.numneigh = c->numneigh;
  a.orig = c->orig;
  a.f = c->f;
  a.partial = c->partial;
  a.counter = c->counter;
  a.ev = c->ev;
  a.eatom = eatom;
  a.vatom = vatom;
  return a;
}

cudaError_t md_rep_step(b200_ctx *c, double dtv, double dtf) {
  const PairArgs a = pair_args(c, nullptr, nullptr);
  RepStepArgs s;
  s.first = c->d_rep_grp_first;
  s.ranges = c->d_rep_ranges;
  s.dtv = dtv;
  s.dtf = dtf;
  s.triggersq = 0.25 * c->skin * c->skin;  // src/neighbor.cpp:239
  s.mass = c->mass_dev;
  s.x4 = c->x4;
  s.v = c->v;
  s.xhold = c->check ? c->xhold : nullptr;
  s.status = c->status;
  s.dcount = c->dec_count;
  s.mail = c->mail_dev;
  s.counter = c->counter;
  s.every = c->every;
  s.delay = c->delay;
  s.check = c->check;
  const bool mixed = c->prec == B200_PREC_MIXED, iso = md_q_iso(c);
  cudaError_t e;
  switch (c->rep_tpa) {
    case 1:
      e = !mixed ? launch_rep_t<1, false, false>(c, a, s)
          : iso  ? launch_rep_t<1, true, true>(c, a, s)
                 : launch_rep_t<1, true, false>(c, a, s);
      break;
    case 2:
      e = !mixed ? launch_rep_t<2, false, false>(c, a, s)
          : iso  ? launch_rep_t<2, true, true>(c, a, s)
                 : launch_rep_t<2, true, false>(c, a, s);
      break;
    default:
      e = !mixed ? launch_rep_t<4, false, false>(c, a, s)
          : iso  ? launch_rep_t<4, true, true>(c, a, s)
                 : launch_rep_t<4, true, false>(c, a, s);
      break;
  }
  c->launches++;
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// Group plan: G = (SMs x CTAs per SM) / cs clusters, at most one per replica;
// replicas go, largest first, to the group with the fewest atoms (longest
// processing time first), so the cluster that finishes last carries about
// the mean load whenever no replica is larger than it.
int md_rep_plan(b200_ctx *c, int cs, int block, int tpa) {
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
  const int per_sm = block <= 256 ? 4 : 2;
  int groups = dev_sms * per_sm / cs;
  if (groups > c->nrep) groups = c->nrep;
  if (groups < 1) groups = 1;
  std::vector<int> order(c->nrep);
  for (int r = 0; r < c->nrep; r++) order[r] = r;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return c->rep_natoms[x] > c->rep_natoms[y]; });
  std::vector<long long> load(groups, 0);
  std::vector<std::vector<int>> members(groups);
  for (int r : order) {
    int best = 0;
    for (int k = 1; k < groups; k++)
      if (load[k] < load[best]) best = k;
    load[best] += c->rep_natoms[r];
    members[best].push_back(r);
  }
  std::vector<int> first(groups + 1, 0);
  std::vector<int2> ranges;
  for (int k = 0; k < groups; k++) {
    std::sort(members[k].begin(), members[k].end());
    for (int r : members[k]) ranges.push_back(make_int2(c->rep_atom_start[r], c->rep_natoms[r]));
    first[k + 1] = (int)ranges.size();
  }
  if (c->d_rep_grp_first) cudaFree(c->d_rep_grp_first);
  if (c->d_rep_ranges) cudaFree(c->d_rep_ranges);
  c->d_rep_grp_first = nullptr;
  c->d_rep_ranges = nullptr;
  cudaError_t e = cudaMalloc((void **)&c->d_rep_grp_first, first.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_rep_ranges, ranges.size() * sizeof(int2));
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_rep_grp_first, first.data(), first.size() * sizeof(int),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_rep_ranges, ranges.data(), ranges.size() * sizeof(int2),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return B200_ERR_CUDA;
  c->rep_cs = cs;
  c->rep_block = block;
  c->rep_tpa = tpa;
  c->rep_groups = groups;
  return B200_OK;
}

cudaError_t md_lj_compute(b200_ctx *c, bool ev, bool atom_ev, double *eatom, double *vatom) {
  PairArgs a;
  a.n = c->n;
  a.stride = c->stride;
  a.ntp1 = c->ntypes + 1;
  a.box = c->box;
  a.reps = c->reps();
  a.tables = c->tables_dev;
  a.cell = c->cell;
  a.nlist = c->nlist;
  a.numneigh = c->numneigh;
  a.orig = c->orig;
  a.f = c->f;
  a.partial = c->partial;
  a.counter = c->counter;
  a.ev = c->ev;
  a.eatom = eatom;
  a.vatom = vatom;
  const bool single = c->ntypes == 1;
  switch (c->tpa) {
    case 1: launch_tpa<1>(c, a, ev, atom_ev, single); break;
    case 2: launch_tpa<2>(c, a, ev, atom_ev, single); break;
    case 4: launch_tpa<4>(c, a, ev, atom_ev, single); break;
    case 8: launch_tpa<8>(c, a, ev, atom_ev, single); break;
    case 16: launch_tpa<16>(c, a, ev, atom_ev, single); break;
    default: launch_tpa<32>(c, a, ev, atom_ev, single); break;
  }
  return cudaGetLastError();
}

// ---- one launch per MD step (k_lj_step) ---------------------------------

namespace {
template <int TPA, bool OUT, bool SINGLE>
void launch_step_t(b200_ctx *c, const PairArgs &a, const StepArgs &s) {
  const int B = 128;
  const int grid = md_blocks((long long)a.n * TPA, B);
  if (c->prec == B200_PREC_MIXED)
    k_lj_step<TPA, OUT, SINGLE, true><<<grid, B, 0, c->stream>>>(a, s);
  else
    k_lj_step<TPA, OUT, SINGLE, false><<<grid, B, 0, c->stream>>>(a, s);
}

template <int TPA>
void launch_step_tpa(b200_ctx *c, const PairArgs &a, const StepArgs &s, bool out) {
  const bool single = c->ntypes == 1;
  if (out) single ? launch_step_t<TPA, true, true>(c, a, s) : launch_step_t<TPA, true, false>(c, a, s);
  else single ? launch_step_t<TPA, false, true>(c, a, s) : launch_step_t<TPA, false, false>(c, a, s);
}
}  // namespace

// One box only: a replica batch keeps its tuned step (the graph of the pair
// kernel and k_nve_fused, or k_rep_step), which measured 5 % faster than
// k_lj_step for the 256-replica batch.
bool md_lj_step_ok(const b200_ctx *c) {
  return c->pstyle == B200_PAIR_LJ_CUT && c->tpa >= 1 && c->tpa <= 8 &&
         (c->prec != B200_PREC_MIXED || md_q_iso(c)) && c->nrep == 0 && !c->ghosts_on;
}

cudaError_t md_lj_step(b200_ctx *c, double dtv, double dtf, bool out) {
  const PairArgs a = pair_args(c, nullptr, nullptr);
  StepArgs s;
  s.dtv = dtv;
  s.dtf = dtf;
  s.triggersq = 0.25 * c->skin * c->skin;  // src/neighbor.cpp:239
  s.mass = c->mass_dev;
  s.x4 = c->x4;
  if (c->prec == B200_PREC_MIXED) {
    s.cur = c->xq;
    s.nxt = c->xqb;
  } else {
    s.cur = c->x4;
    s.nxt = c->x4b;
  }
  s.v = c->v;
  s.xhold = c->check ? c->xhold : nullptr;
  s.status = c->status;
  s.dcount = c->dec_count;
  s.mail = c->mail_dev;
  s.rows = c->rows;
  s.rows_cap = c->rows_cap;
  s.every = c->every;
  s.delay = c->delay;
  s.check = c->check;
  switch (c->tpa) {
    case 1: launch_step_tpa<1>(c, a, s, out); break;
    case 2: launch_step_tpa<2>(c, a, s, out); break;
    case 4: launch_step_tpa<4>(c, a, s, out); break;
    default: launch_step_tpa<8>(c, a, s, out); break;
  }
  c->launches++;
  cudaError_t e = cudaGetLastError();
  // the next step's rebuild decision (an output step's last block made it)
  if (e == cudaSuccess && !out) e = md_decide(c);
  return e;
}

void md_swap_positions(b200_ctx *c) {
  if (c->prec == B200_PREC_MIXED) std::swap(c->xq, c->xqb);
  else std::swap(c->x4, c->x4b);
  c->pos_parity ^= 1;
}
