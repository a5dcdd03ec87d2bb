// pair_eam.cu -- pair_style eam / eam/alloy / eam/fs over the full list.
//
// Replaces PairEAM::compute (src/MANYBODY/pair_eam.cpp:125-306), whose three
// passes become two kernels:
//   k_eam_rho    density rho_i over the full list (no ghost densities, so the
//                reverse_comm_pair of rho disappears) and, in the same
//                kernel, the embedding derivative fp_i = F'(rho_i) and energy
//                F(rho_i) (+ linear term above rhomax)            (:160-228)
//   k_eam_force  pair force psi'/r using fp_i and the neighbor's own fp_j
//                (the forward_comm_pair of fp disappears)         (:237-303)
// Splines are the reference's 7-coefficient cubic tables
// (PairEAM::interpolate, :723-751), stored 8 doubles per knot (density and
// pair rows reordered [c3 c4 c5 c6 | c0 c1 c2 -] so the value and the
// derivative coefficients are each 16-byte loads; embedding rows as
// [c0..c6 -]); the index
// clamps are the reference's: m = min(m, nr-1), p = min(p, 1) for r and
// m = max(1, min(m, nrho-1)) for rho.
// Mixed form: FP32 tables reordered per knot as [c3 c4 c5 c6 | c0 c1 c2 -]
// so one float4 load gives a value and one a derivative; separations from the
// fixed-point coordinates (md_xq: one 32-bit subtraction and one conversion
// per component, at the minimum image); fp_j gathered as FP32; sums in FP64.  The
// embedding step F(rho) stays FP64 in both forms.  Each thread reads four
// list entries with one 16-byte load and issues their gathers together; the
// mixed kernels load the next slab's entries before using the current one.
// With one element the mixed force kernel reads each knot's z2 value and
// rho' coefficients as one 32-byte record (fz_f) and forms the z2
// derivative from the value coefficients, (3 c3 p^2 + 2 c4 p + c5) / dr,
// the relation PairEAM::interpolate (:723-751) builds the stored derivative
// coefficients from.
#include "md_state.h"

namespace {

struct EamArgs {
  int n, stride, ntp1;
  BoxGeom box;
  const int *cell, *nlist, *numneigh, *orig;
  int nrho, nr;
  bool rhor_sym;  // rho'_j spline row == rho'_i spline row for every pair
  double rdr, rdrho, rhomax, cutforcesq;
  const double *frho, *rhor, *z2r;
  const float *rhor_f, *z2r_f;
  const float *fz_f;  // one element: per knot [z2 c3 c4 c5 c6 | rho' c0 c1 c2 | 0]
  const int *t2frho, *t2rhor, *t2z2r;  // device copies of the type maps
  double *rho, *fp;
  float *fpf;
  double *f;
  double *partial;
  unsigned int *counter;
  double *ev;
  double *eatom, *vatom;
  StepArgs step;  // k_eam_force with STEP: the half-steps after the forces
};

__device__ __forceinline__ void decode(unsigned int e, int &j, int &dx, int &dy, int &dz) {
  md_entry(e, j, dx, dy, dz);
}

// Spline knot and fraction of the mixed form from p = x * rdx + 1 >= 1:
// m = min(floor(p), mmax), frac = min(p - m, 1) -- the reference's
// static_cast<int> truncation (equal to floor here, p > 0) and clamps.  The
// floor comes from a round-down add of 2^23, which leaves floor(p) in the
// low mantissa bits (exact for p < 2^23), instead of float-to-integer and
// integer-to-float conversions.
__device__ __forceinline__ void knot_f(float p, int mmax, int &m, float &frac) {
  const float t = __fadd_rd(p, 8388608.0f);
  m = min(__float_as_int(t) - 0x4B000000, mmax);
  frac = fminf(p - fminf(t - 8388608.0f, (float)mmax), 1.0f);
}

// The same for the FP64 form: floor(p) from a round-down add of 2^52 (exact
// for p < 2^52), and p - m exactly as the reference's p -= m.
__device__ __forceinline__ void knot_d(double p, int mmax, int &m, double &frac) {
  const double t = __dadd_rd(p, 4503599627370496.0);
  m = min((int)(__double_as_longlong(t) - 0x4330000000000000LL), mmax);
  frac = fmin(p - (double)m, 1.0);
}

// Embedding F(rho) and F'(rho) of one atom, FP64, reference clamps.
__device__ __forceinline__ void embed(const EamArgs &a, int itype_frho, double rho, double &fp,
                                      double &phi) {
  double p = __dadd_rn(__dmul_rn(rho, a.rdrho), 1.0);
  int m = (int)p;
  m = max(1, min(m, a.nrho - 1));
  p -= m;
  p = fmin(p, 1.0);
  const double *c = a.frho + ((size_t)itype_frho * (a.nrho + 1) + m) * 8;
  fp = (c[0] * p + c[1]) * p + c[2];
  phi = ((c[3] * p + c[4]) * p + c[5]) * p + c[6];
  if (rho > a.rhomax) phi += fp * (rho - a.rhomax);
}

template <int TPA, bool EV, bool ATOM, bool MIXED, bool SINGLE>
__global__ void __launch_bounds__(128) k_eam_rho(EamArgs a, const double4 *__restrict__ x4,
                                                 const int4 *__restrict__ xq) {
  __shared__ int s_t2rhor[TABSZ];
  __shared__ int s_t2frho[MD_MAXTYPES + 1];
  __shared__ double red[7 * 4];
  const int nt2 = a.ntp1 * a.ntp1;
  for (int k = threadIdx.x; k < nt2; k += blockDim.x) s_t2rhor[k] = a.t2rhor[k];
  for (int k = threadIdx.x; k < a.ntp1; k += blockDim.x) s_t2frho[k] = a.t2frho[k];
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / TPA, lane = t % TPA;
  const bool active = i < a.n;
  double rho = 0.0;
  int ti = 1;
  if (active) {
    const int num = a.numneigh[i];
    if (!MIXED) {
      const double4 xi = x4[i];
      ti = (int)xi.w;
      int cx, cy, cz;
      md_cell_unpack(a.cell[i], cx, cy, cz);
      const Shift3 sx = shifts(cx, a.box.ncell[0], a.box.prd[0]);
      const Shift3 sy = shifts(cy, a.box.ncell[1], a.box.prd[1]);
      const Shift3 sz = shifts(cz, a.box.ncell[2], a.box.prd[2]);
      // one element: the density spline row of every pair
      const double *rrow =
          SINGLE ? a.rhor + (size_t)s_t2rhor[a.ntp1 + 1] * (a.nr + 1) * 8 : nullptr;
      // four entries ee of this lane (walk_list); the first mm lie before the
      // atom's count
      auto four = [&](const unsigned (&ee)[4], int mm) {
        double4 xq[4];
#pragma unroll
        for (int u = 0; u < 4; u++) xq[u] = x4[u < mm ? md_entry_j(ee[u]) : i];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (u >= mm) break;
          int j, dx, dy, dz;
          decode(ee[u], j, dx, dy, dz);
          const double4 xj = xq[u];
          const double delx = __dsub_rn(xi.x, __dadd_rn(xj.x, pick(sx, dx)));
          const double dely = __dsub_rn(xi.y, __dadd_rn(xj.y, pick(sy, dy)));
          const double delz = __dsub_rn(xi.z, __dadd_rn(xj.z, pick(sz, dz)));
          const double rsq = dsq3(delx, dely, delz);
          if (rsq < a.cutforcesq) {
            int m;
            double p;
            knot_d(__dadd_rn(__dmul_rn(sqrt(rsq), a.rdr), 1.0), a.nr - 1, m, p);
            const double *row =
                SINGLE ? rrow : a.rhor + (size_t)s_t2rhor[(int)xj.w * a.ntp1 + ti] * (a.nr + 1) * 8;
            // knot layout [c3 c4 c5 c6 | c0 c1 c2 -]: the value coefficients
            // are two 16-byte loads
            const double2 v01 = __ldg(reinterpret_cast<const double2 *>(row + (size_t)m * 8));
            const double2 v23 = __ldg(reinterpret_cast<const double2 *>(row + (size_t)m * 8 + 2));
            rho += ((v01.x * p + v01.y) * p + v23.x) * p + v23.y;
          }
        }
      };
      walk_list<TPA>(a.nlist, a.stride, i, num, lane, four);
    } else {
      const int4 xi = xq[i];
      ti = xi.w;
      const float qx = a.box.qs[0], qy = a.box.qs[1], qz = a.box.qs[2];
      const float qxl = a.box.qs_lo[0], qyl = a.box.qs_lo[1], qzl = a.box.qs_lo[2];
      const float cutf = (float)a.cutforcesq, rdrf = (float)a.rdr;
      // one element: the density spline row of every pair
      const float *rrow =
          SINGLE ? a.rhor_f + (size_t)s_t2rhor[a.ntp1 + 1] * (a.nr + 1) * 8 : nullptr;
      // four entries ee of this lane (walk_list)
      auto four = [&](const unsigned (&ee)[4], int) {
        // whole slabs: pad entries in the last slab name the atom itself
        // (zero separation), which the r^2 > 0 test rejects
        int4 xs[4];
#pragma unroll
        for (int u = 0; u < 4; u++) xs[u] = xq[md_entry_j(ee[u])];
        float crho = 0.f;  // FP32 slab sum, added to the FP64 density
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int4 xj = xs[u];
          // minimum-image separation from the fixed-point coordinates
          const float delx = md_qlen(md_qdiff(xi.x, xj.x), qx, qxl);
          const float dely = md_qlen(md_qdiff(xi.y, xj.y), qy, qyl);
          const float delz = md_qlen(md_qdiff(xi.z, xj.z), qz, qzl);
          const float rsq = delx * delx + dely * dely + delz * delz;
          if (rsq < cutf && rsq > 0.f) {
            int m;
            float p;
            knot_f(rsq * rsqrtf(rsq) * rdrf + 1.0f, a.nr - 1, m, p);
            const float *row = SINGLE ? rrow
                                      : a.rhor_f + (size_t)s_t2rhor[xj.w * a.ntp1 + ti] *
                                                       (a.nr + 1) * 8;
            const float4 c = __ldg(reinterpret_cast<const float4 *>(row + (size_t)m * 8));
            crho += ((c.x * p + c.y) * p + c.z) * p + c.w;
          }
        }
        rho += (double)crho;
      };
      walk_list<TPA>(a.nlist, a.stride, i, num, lane, four);
    }
  }
  rho = lane_sum<TPA>(rho);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (active && lane == 0) {
    double fpi, phi;
    embed(a, s_t2frho[ti], rho, fpi, phi);
    a.rho[i] = rho;
    a.fp[i] = fpi;
    if (MIXED) a.fpf[i] = (float)fpi;
    if (EV) {
      acc[0] = phi;
      if (ATOM && a.eatom) a.eatom[a.orig[i]] = phi;
    }
  }
  if (EV) block_partials_finish<7>(acc, red, a.partial, a.counter, a.ev, false);
}

// STEP: a one-launch step (md_step_atom / md_step_tail): after the forces
// each atom's first lane applies this step's final half-step and the next
// step's initial half-step, writing the new positions to the other buffer.
template <int TPA, bool EV, bool ATOM, bool MIXED, bool SINGLE, bool STEP = false>
__global__ void __launch_bounds__(128) k_eam_force(EamArgs a, const double4 *__restrict__ x4,
                                                   const int4 *__restrict__ xq) {
  __shared__ int s_t2rhor[TABSZ];
  __shared__ int s_t2z2r[TABSZ];
  __shared__ double red[8 * 4];
  const int nt2 = a.ntp1 * a.ntp1;
  for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
    s_t2rhor[k] = a.t2rhor[k];
    s_t2z2r[k] = a.t2z2r[k];
  }
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / TPA, lane = t % TPA;
  const bool active = i < a.n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (active) {
    const int num = a.numneigh[i];
    if (!MIXED) {
      const double4 xi = x4[i];
      const int ti = (int)xi.w;
      const double fpi = a.fp[i];
      int cx, cy, cz;
      md_cell_unpack(a.cell[i], cx, cy, cz);
      const Shift3 sx = shifts(cx, a.box.ncell[0], a.box.prd[0]);
      const Shift3 sy = shifts(cy, a.box.ncell[1], a.box.prd[1]);
      const Shift3 sz = shifts(cz, a.box.ncell[2], a.box.prd[2]);
      // one element: the density and pair spline rows of every pair
      const double *rrow1 =
          SINGLE ? a.rhor + (size_t)s_t2rhor[a.ntp1 + 1] * (a.nr + 1) * 8 : nullptr;
      const double *zrow1 = SINGLE ? a.z2r + (size_t)s_t2z2r[a.ntp1 + 1] * (a.nr + 1) * 8 : nullptr;
      // four entries ee of this lane (walk_list); the first mm lie before the
      // atom's count
      auto four = [&](const unsigned (&ee)[4], int mm) {
       double4 xq[4];
       double fpq[4];
#pragma unroll
       for (int u = 0; u < 4; u++) {
         const int jj = u < mm ? md_entry_j(ee[u]) : i;
         xq[u] = x4[jj];
         fpq[u] = a.fp[jj];
       }
#pragma unroll
       for (int u = 0; u < 4; u++) {
        if (u >= mm) break;
        int j, dx, dy, dz;
        decode(ee[u], j, dx, dy, dz);
        const double4 xj = xq[u];
        const double delx = __dsub_rn(xi.x, __dadd_rn(xj.x, pick(sx, dx)));
        const double dely = __dsub_rn(xi.y, __dadd_rn(xj.y, pick(sy, dy)));
        const double delz = __dsub_rn(xi.z, __dadd_rn(xj.z, pick(sz, dz)));
        const double rsq = dsq3(delx, dely, delz);
        if (rsq < a.cutforcesq) {
          const int tj = (int)xj.w;
          const double r = sqrt(rsq);
          int m;
          double p;
          knot_d(__dadd_rn(__dmul_rn(r, a.rdr), 1.0), a.nr - 1, m, p);
          const size_t o8 = (size_t)m * 8;
          // knot layout [c3 c4 c5 c6 | c0 c1 c2 -]
          const double *ci =
              (SINGLE ? rrow1 : a.rhor + (size_t)s_t2rhor[ti * a.ntp1 + tj] * (a.nr + 1) * 8) + o8;
          const double2 d01 = __ldg(reinterpret_cast<const double2 *>(ci + 4));
          const double rhoip = (d01.x * p + d01.y) * p + __ldg(ci + 6);
          double rhojp = rhoip;
          if (!SINGLE && !a.rhor_sym) {
            const double *cj = a.rhor + ((size_t)s_t2rhor[tj * a.ntp1 + ti] * (a.nr + 1) + m) * 8;
            const double2 e01 = __ldg(reinterpret_cast<const double2 *>(cj + 4));
            rhojp = (e01.x * p + e01.y) * p + __ldg(cj + 6);
          }
          const double *cz2 =
              (SINGLE ? zrow1 : a.z2r + (size_t)s_t2z2r[ti * a.ntp1 + tj] * (a.nr + 1) * 8) + o8;
          const double2 z01 = __ldg(reinterpret_cast<const double2 *>(cz2));
          const double2 z23 = __ldg(reinterpret_cast<const double2 *>(cz2 + 2));
          const double2 zd01 = __ldg(reinterpret_cast<const double2 *>(cz2 + 4));
          const double z2p = (zd01.x * p + zd01.y) * p + __ldg(cz2 + 6);
          const double z2 = ((z01.x * p + z01.y) * p + z23.x) * p + z23.y;
          const double recip = rcp_nr(r);
          const double phi = z2 * recip;
          const double phip = z2p * recip - phi * recip;
          const double psip = fpi * rhojp + fpq[u] * rhoip + phip;
          const double fpair = -psip * recip;
          fx += delx * fpair;
          fy += dely * fpair;
          fz += delz * fpair;
          if (EV) {
            acc[0] += 0.5 * phi;
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
      walk_list<TPA>(a.nlist, a.stride, i, num, lane, four);
    } else {
      const int4 xi = xq[i];
      const int ti = xi.w;
      const float fpi = a.fpf[i];
      const float qx = a.box.qs[0], qy = a.box.qs[1], qz = a.box.qs[2];
      const float qxl = a.box.qs_lo[0], qyl = a.box.qs_lo[1], qzl = a.box.qs_lo[2];
      const float cutf = (float)a.cutforcesq, rdrf = (float)a.rdr;
      // one element: the density-derivative and pair spline rows of every pair
      const float *drow1 = SINGLE ? a.fz_f + 4 : nullptr;
      const float *zrow1 = SINGLE ? a.fz_f : nullptr;
      // four entries ee of this lane (walk_list)
      auto four = [&](const unsigned (&ee)[4], int) {
       // whole slabs: pad entries in the last slab name the atom itself
       // (zero separation), which the r^2 > 0 test rejects
       int4 xs[4];
       float fpq[4];
#pragma unroll
       for (int u = 0; u < 4; u++) {
         const int jj = md_entry_j(ee[u]);
         xs[u] = xq[jj];
         fpq[u] = a.fpf[jj];
       }
       // FP32 sum of the slab's pair forces, added to the FP64 accumulator
       float cfx = 0.f, cfy = 0.f, cfz = 0.f;
       float ce[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // EV: the slab's FP32 sums
#pragma unroll
       for (int u = 0; u < 4; u++) {
        const int4 xj = xs[u];
        // minimum-image separation from the fixed-point coordinates
        const float delx = md_qlen(md_qdiff(xi.x, xj.x), qx, qxl);
        const float dely = md_qlen(md_qdiff(xi.y, xj.y), qy, qyl);
        const float delz = md_qlen(md_qdiff(xi.z, xj.z), qz, qzl);
        const float rsq = delx * delx + dely * dely + delz * delz;
        if (rsq < cutf && rsq > 0.f) {
          const int tj = xj.w;
          const float recip = rsqrtf(rsq);
          const float r = rsq * recip;
          int m;
          float p;
          knot_f(r * rdrf + 1.0f, a.nr - 1, m, p);
          const size_t o8 = (size_t)m * 8;
          const float *drow =
              SINGLE ? drow1 : a.rhor_f + (size_t)s_t2rhor[ti * a.ntp1 + tj] * (a.nr + 1) * 8 + 4;
          const float4 ci = __ldg(reinterpret_cast<const float4 *>(drow + o8));
          const float rhoip = (ci.x * p + ci.y) * p + ci.z;
          float rhojp = rhoip;
          if (!SINGLE && !a.rhor_sym) {
            const float4 cj = __ldg(reinterpret_cast<const float4 *>(
                a.rhor_f + ((size_t)s_t2rhor[tj * a.ntp1 + ti] * (a.nr + 1) + m) * 8 + 4));
            rhojp = (cj.x * p + cj.y) * p + cj.z;
          }
          const float *zb =
              (SINGLE ? zrow1 : a.z2r_f + (size_t)s_t2z2r[ti * a.ntp1 + tj] * (a.nr + 1) * 8) + o8;
          const float4 zv = __ldg(reinterpret_cast<const float4 *>(zb));
          float z2p;
          if (SINGLE) {
            // the z2 derivative from the value coefficients:
            // (3 c3 p^2 + 2 c4 p + c5) / dr, as PairEAM::interpolate stores it
            z2p = (fmaf(3.0f * zv.x, p, 2.0f * zv.y) * p + zv.z) * rdrf;
          } else {
            const float4 zd = __ldg(reinterpret_cast<const float4 *>(zb + 4));
            z2p = (zd.x * p + zd.y) * p + zd.z;
          }
          const float z2 = ((zv.x * p + zv.y) * p + zv.z) * p + zv.w;
          const float phi = z2 * recip;
          const float phip = z2p * recip - phi * recip;
          const float psip = fpi * rhojp + fpq[u] * rhoip + phip;
          const float fpair = -psip * recip;
          cfx += delx * fpair;
          cfy += dely * fpair;
          cfz += delz * fpair;
          if (EV) {
            ce[0] = fmaf(0.5f, phi, ce[0]);
            const float hf = 0.5f * fpair;
            ce[1] = fmaf(delx * delx, hf, ce[1]);
            ce[2] = fmaf(dely * dely, hf, ce[2]);
            ce[3] = fmaf(delz * delz, hf, ce[3]);
            ce[4] = fmaf(delx * dely, hf, ce[4]);
            ce[5] = fmaf(delx * delz, hf, ce[5]);
            ce[6] = fmaf(dely * delz, hf, ce[6]);
          }
        }
       }
       fx += (double)cfx;
       fy += (double)cfy;
       fz += (double)cfz;
       // the energy and virial terms join the FP64 sums once per slab, as the
       // forces do
       if (EV)
#pragma unroll
         for (int k = 0; k < 7; k++) acc[k] += (double)ce[k];
      };
      walk_list<TPA>(a.nlist, a.stride, i, num, lane, four);
    }
  }
  fx = lane_sum<TPA>(fx);
  fy = lane_sum<TPA>(fy);
  fz = lane_sum<TPA>(fz);
  if (STEP) {
    double ke = 0.0;
    bool moved = false;
    if (active && lane == 0)
      moved = md_step_atom<EV, MIXED>(a.step, i, a.stride, a.f, fx, fy, fz, a.box, ke);
    // ev[0..6] already hold the density pass's embedding energy: add to it
    md_step_tail<EV>(a.step, moved, acc, ke, red, a.partial, a.counter, a.ev, true);
    return;
  }
  if (active && lane == 0) {
    a.f[i] = fx;
    a.f[a.stride + i] = fy;
    a.f[2 * a.stride + i] = fz;
  }
  if (EV) {
    if (ATOM) {
      double e[7];
#pragma unroll
      for (int k = 0; k < 7; k++) e[k] = lane_sum<TPA>(acc[k]);
      if (active && lane == 0) {
        const int o = a.orig[i];
        if (a.eatom) a.eatom[o] += e[0];
        if (a.vatom)
#pragma unroll
          for (int k = 0; k < 6; k++) a.vatom[6 * (size_t)o + k] = e[1 + k];
      }
    }
    block_partials_finish<7>(acc, red, a.partial, a.counter, a.ev, true);
  }
}

// phase event between the two passes: an event-record node when the stream
// is being captured into a step graph, a plain record otherwise
void record_mid(b200_ctx *c, cudaEvent_t mid) {
  if (!mid) return;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(c->stream, &st);
  if (st == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(mid, c->stream, cudaEventRecordExternal);
  else
    cudaEventRecord(mid, c->stream);
}

// stage: EAM_BOTH, or EAM_DENSITY (passes 1-2) / EAM_FORCE (pass 3) alone
template <int TPA, bool EV, bool ATOM, bool SINGLE>
void launch_t(b200_ctx *c, const EamArgs &a, cudaEvent_t mid, int stage, bool step = false) {
  const int B = 128;
  const int grid = md_blocks((long long)a.n * TPA, B);
  if (stage != EAM_FORCE) {
    if (c->prec == B200_PREC_MIXED)
      k_eam_rho<TPA, EV, ATOM, true, SINGLE><<<grid, B, 0, c->stream>>>(a, c->x4, c->xq);
    else
      k_eam_rho<TPA, EV, ATOM, false, SINGLE><<<grid, B, 0, c->stream>>>(a, c->x4, c->xq);
    c->launches++;
  }
  record_mid(c, mid);
  if (stage != EAM_DENSITY) {
    if constexpr (!ATOM) {
      if (step) {
        if (c->prec == B200_PREC_MIXED)
          k_eam_force<TPA, EV, false, true, SINGLE, true><<<grid, B, 0, c->stream>>>(a, c->x4, c->xq);
        else
          k_eam_force<TPA, EV, false, false, SINGLE, true><<<grid, B, 0, c->stream>>>(a, c->x4,
                                                                                      c->xq);
        c->launches++;
        return;
      }
    }
    if (c->prec == B200_PREC_MIXED)
      k_eam_force<TPA, EV, ATOM, true, SINGLE><<<grid, B, 0, c->stream>>>(a, c->x4, c->xq);
    else
      k_eam_force<TPA, EV, ATOM, false, SINGLE><<<grid, B, 0, c->stream>>>(a, c->x4, c->xq);
    c->launches++;
  }
}

template <int TPA, bool SINGLE>
void launch_ts(b200_ctx *c, const EamArgs &a, bool ev, bool atom, cudaEvent_t mid, int stage) {
  if (!ev) launch_t<TPA, false, false, SINGLE>(c, a, mid, stage);
  else if (!atom) launch_t<TPA, true, false, SINGLE>(c, a, mid, stage);
  else launch_t<TPA, true, true, SINGLE>(c, a, mid, stage);
}

template <int TPA>
void launch_tpa(b200_ctx *c, const EamArgs &a, bool ev, bool atom, cudaEvent_t mid, int stage) {
  // one element type: spline rows hoisted out of the pair loop (mixed form)
  if (c->ntypes == 1) launch_ts<TPA, true>(c, a, ev, atom, mid, stage);
  else launch_ts<TPA, false>(c, a, ev, atom, mid, stage);
}

// F'(rho) of caller atoms idx[i] into / from buf[i] (PairEAM::pack_forward_comm
// / unpack_forward_comm, src/MANYBODY/pair_eam.cpp:809-831); unpack also
// sets the FP32 copy the mixed force pass reads
__global__ void k_fp_pack(int m, int n, const int *__restrict__ idx, const int *__restrict__ where,
                          const double *__restrict__ fp, double *__restrict__ buf,
                          int *__restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int j = idx[i];
  if (j < 0 || j >= n) {
    atomicExch(&status[ST_HALO_BAD], 1);
    return;
  }
  buf[i] = fp[where[j]];
}

__global__ void k_fp_unpack(int m, int n, const int *__restrict__ idx,
                            const int *__restrict__ where, const int *__restrict__ ghost,
                            const double *__restrict__ buf, double *__restrict__ fp,
                            float *__restrict__ fpf, int *__restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int j = idx[i];
  if (j < 0 || j >= n) {
    atomicExch(&status[ST_HALO_BAD], 1);
    return;
  }
  if (ghost && ghost[j] == 0) {  // owned atoms keep their own F'
    atomicExch(&status[ST_HALO_BAD], 2);
    return;
  }
  const int k = where[j];
  fp[k] = buf[i];
  if (fpf) fpf[k] = (float)buf[i];
}

}  // namespace

cudaError_t md_eam_fp_halo(b200_ctx *c, int m, const int *idx, double *buf, bool pack) {
  if (m < 1) return cudaSuccess;
  if (pack)
    k_fp_pack<<<md_blocks(m, 256), 256, 0, c->stream>>>(m, c->n, idx, c->where, c->fp, buf,
                                                        c->status);
  else
    k_fp_unpack<<<md_blocks(m, 256), 256, 0, c->stream>>>(
        m, c->n, idx, c->where, c->ghosts_on ? c->ghost : nullptr, buf, c->fp,
        c->prec == B200_PREC_MIXED ? c->fpf : nullptr, c->status);
  c->launches++;
  return cudaGetLastError();
}

static EamArgs eam_args(b200_ctx *c, double *eatom, double *vatom) {
  EamArgs a;
  a.n = c->n;
  a.stride = c->stride;
  a.ntp1 = c->ntypes + 1;
  a.box = c->box;
  a.cell = c->cell;
  a.nlist = c->nlist;
  a.numneigh = c->numneigh;
  a.orig = c->orig;
  a.nrho = c->eam.nrho;
  a.nr = c->eam.nr;
  a.rhor_sym = c->eam.rhor_sym;
  a.rdr = c->eam.rdr;
  a.rdrho = c->eam.rdrho;
  a.rhomax = c->eam.rhomax;
  a.cutforcesq = c->eam.cutforcesq;
  a.frho = c->eam.frho;
  a.rhor = c->eam.rhor;
  a.z2r = c->eam.z2r;
  a.rhor_f = c->eam.rhor_f;
  a.z2r_f = c->eam.z2r_f;
  a.fz_f = c->eam.fz_f;
  // type maps live right after the TAB_* tables in tables_dev (as ints)
  const int *maps = reinterpret_cast<const int *>(c->tables_dev + TAB_COUNT * TABSZ);
  a.t2frho = maps;
  a.t2rhor = maps + (MD_MAXTYPES + 1);
  a.t2z2r = maps + (MD_MAXTYPES + 1) + TABSZ;
  a.rho = c->rho;
  a.fp = c->fp;
  a.fpf = c->fpf;
  a.f = c->f;
  a.partial = c->partial;
  a.counter = c->counter;
  a.ev = c->ev;
  a.eatom = eatom;
  a.vatom = vatom;
  return a;
}

cudaError_t md_eam_compute(b200_ctx *c, bool ev, bool atom_ev, double *eatom, double *vatom,
                           cudaEvent_t mid, int stage) {
  EamArgs a = eam_args(c, eatom, vatom);
  switch (c->tpa) {
    case 1: launch_tpa<1>(c, a, ev, atom_ev, mid, stage); break;
    case 2: launch_tpa<2>(c, a, ev, atom_ev, mid, stage); break;
    case 4: launch_tpa<4>(c, a, ev, atom_ev, mid, stage); break;
    case 8: launch_tpa<8>(c, a, ev, atom_ev, mid, stage); break;
    case 16: launch_tpa<16>(c, a, ev, atom_ev, mid, stage); break;
    default: launch_tpa<32>(c, a, ev, atom_ev, mid, stage); break;
  }
  return cudaGetLastError();
}

// ---- one launch per EAM force pass and half-steps --------------------------

namespace {
template <int TPA>
void launch_step_tpa(b200_ctx *c, const EamArgs &a, bool out) {
  if (c->ntypes == 1) {
    if (out) launch_t<TPA, true, false, true>(c, a, nullptr, EAM_BOTH, true);
    else launch_t<TPA, false, false, true>(c, a, nullptr, EAM_BOTH, true);
  } else {
    if (out) launch_t<TPA, true, false, false>(c, a, nullptr, EAM_BOTH, true);
    else launch_t<TPA, false, false, false>(c, a, nullptr, EAM_BOTH, true);
  }
}
}  // namespace

bool md_eam_step_ok(const b200_ctx *c) {
  return c->pstyle == B200_PAIR_EAM && c->tpa >= 1 && c->tpa <= 8 && c->nrep == 0 &&
         !c->ghosts_on;
}

cudaError_t md_eam_step(b200_ctx *c, double dtv, double dtf, bool out) {
  EamArgs a = eam_args(c, nullptr, nullptr);
  StepArgs &s = a.step;
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
    case 1: launch_step_tpa<1>(c, a, out); break;
    case 2: launch_step_tpa<2>(c, a, out); break;
    case 4: launch_step_tpa<4>(c, a, out); break;
    default: launch_step_tpa<8>(c, a, out); break;
  }
  cudaError_t e = cudaGetLastError();
  // the next step's rebuild decision (an output step's last block made it)
  if (e == cudaSuccess && !out) e = md_decide(c);
  return e;
}
