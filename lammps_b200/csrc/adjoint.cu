// adjoint.cu -- forces and their adjoint for differentiable force matching
// with pair_style lj/cut (any number of types up to MD_ADJ_MAXTYPES).
//
// Forward:  F_i = sum_j phi_ij d_ij,  d_ij = x_i - x_j (periodic image),
//           phi = (lj1 r^-6 - lj2) r^-6 r^-2  for r^2 < cutsq[ti][tj]
//           -- the pair force of PairLJCut::compute (src/pair_lj_cut.cpp:100-113)
//           with lj1 = 48 eps sigma^12, lj2 = 24 eps sigma^6
//           (PairLJCut::init_one, src/pair_lj_cut.cpp:560-563).
// Backward, given G = dL/dF (per atom):
//   dL/dlj1[ti][tj] = sum over directed pairs (G_i . d_ij) r^-14
//   dL/dlj2[ti][tj] = -sum over directed pairs (G_i . d_ij) r^-8
//   dL/dx_i = sum_j H_ij (G_i - G_j),  H_ij = phi I + 2 phi' d d^T,
//             phi' = dphi/d(r^2) = (4 lj2 - 7 lj1 r^-6) r^-6 r^-4
// (the Hessian-vector product of the loss through the forces).  With the
// engine's full neighbor list every atom sums its own terms, so neither pass
// needs atomics; per-type-pair parameter gradients are reduced per block and
// then in a fixed order, so results are reproducible.  The cutoff itself is
// not differentiated: a pair that crosses r = rc under a parameter change
// contributes a jump that finite differences see and this gradient does not.
//
// MIXED: FP32 pair arithmetic on separations formed from the fixed-point
// coordinates (md_xq, as the mixed force kernels), FP64 accumulation of
// forces, gradients and sums.
#include "md_state.h"

namespace {

constexpr int kAdjThreads = 128;
constexpr int kAdjNP = MD_ADJ_MAXTYPES * MD_ADJ_MAXTYPES;  // type pairs

struct AdjTables {
  int ntypes;
  double lj1[kAdjNP], lj2[kAdjNP], cutsq[kAdjNP];  // [(ti-1)*ntypes + (tj-1)]
};

template <bool MIXED>
__device__ __forceinline__ void pair_geom(const AdjTables &T, int i, unsigned e,
                                          const double4 *__restrict__ x4,
                                          const int4 *__restrict__ xq, const Shift3 &sx,
                                          const Shift3 &sy, const Shift3 &sz, const float *qh,
                                          const float *ql, double &dx, double &dy,
                                          double &dz, double &rsq, int &tt) {
  const int j = md_entry_j(e);
  if (MIXED) {
    // minimum-image separation from the fixed-point coordinates
    const int4 xi = xq[i], xj = xq[j];
    const float fx = md_qlen(md_qdiff(xi.x, xj.x), qh[0], ql[0]);
    const float fy = md_qlen(md_qdiff(xi.y, xj.y), qh[1], ql[1]);
    const float fz = md_qlen(md_qdiff(xi.z, xj.z), qh[2], ql[2]);
    dx = fx;
    dy = fy;
    dz = fz;
    rsq = (double)(fx * fx + fy * fy + fz * fz);
    tt = (xi.w - 1) * T.ntypes + (xj.w - 1);
  } else {
    const double4 xi = x4[i], xj = x4[j];
    int jj, ex, ey, ez;
    md_entry(e, jj, ex, ey, ez);
    dx = xi.x - (xj.x + pick(sx, ex));
    dy = xi.y - (xj.y + pick(sy, ey));
    dz = xi.z - (xj.z + pick(sz, ez));
    rsq = dx * dx + dy * dy + dz * dz;
    tt = ((int)xi.w - 1) * T.ntypes + ((int)xj.w - 1);
  }
}

// forces in the caller's order: f[3*orig[i] + k]
template <bool MIXED>
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_forward(int n, int stride, AdjTables T, BoxGeom box, const double4 *__restrict__ x4,
                  const int4 *__restrict__ xq, const int *__restrict__ cell,
                  const int *__restrict__ nlist, const int *__restrict__ numneigh,
                  const int *__restrict__ orig, double *__restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int cx, cy, cz;
  md_cell_unpack(cell[i], cx, cy, cz);
  const Shift3 sx = shifts(cx, box.ncell[0], box.prd[0]);
  const Shift3 sy = shifts(cy, box.ncell[1], box.prd[1]);
  const Shift3 sz = shifts(cz, box.ncell[2], box.prd[2]);
  const int num = numneigh[i];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int k = 0; k < num; k++) {
    const unsigned e = (unsigned)nlist[md_slab(k, i, stride)];
    double dx, dy, dz, rsq;
    int tt;
    pair_geom<MIXED>(T, i, e, x4, xq, sx, sy, sz, box.qs, box.qs_lo, dx, dy, dz, rsq, tt);
    if (rsq < T.cutsq[tt]) {
      double phi;
      if (MIXED) {
        const float r2i = 1.0f / (float)rsq, r6i = r2i * r2i * r2i;
        phi = (double)(((float)T.lj1[tt] * r6i - (float)T.lj2[tt]) * r6i * r2i);
      } else {
        const double r2i = 1.0 / rsq, r6i = r2i * r2i * r2i;
        phi = (T.lj1[tt] * r6i - T.lj2[tt]) * r6i * r2i;
      }
      fx += phi * dx;
      fy += phi * dy;
      fz += phi * dz;
    }
  }
  const int o = orig[i];
  f[3 * o] = fx;
  f[3 * o + 1] = fy;
  f[3 * o + 2] = fz;
}

// G in the caller's order -> G in the sorted order
__global__ void k_adj_gather(int n, const int *__restrict__ orig, const double *__restrict__ g,
                             double *__restrict__ gs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = orig[i];
  gs[3 * i] = g[3 * o];
  gs[3 * i + 1] = g[3 * o + 1];
  gs[3 * i + 2] = g[3 * o + 2];
}

template <bool MIXED>
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_backward(int n, int stride, AdjTables T, BoxGeom box, const double4 *__restrict__ x4,
                   const int4 *__restrict__ xq, const int *__restrict__ cell,
                   const int *__restrict__ nlist, const int *__restrict__ numneigh,
                   const int *__restrict__ orig, const double *__restrict__ gs,
                   double *__restrict__ gx, double *partial, unsigned int *counter,
                   double *gtab) {
  __shared__ double red[2 * kAdjNP * (kAdjThreads / 32)];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // per type pair: dL/dlj1, dL/dlj2 (selected by a compile-time unrolled
  // loop so the accumulators stay in registers)
  double acc[2 * kAdjNP];
#pragma unroll
  for (int k = 0; k < 2 * kAdjNP; k++) acc[k] = 0.0;
  if (i < n) {
    int cx, cy, cz;
    md_cell_unpack(cell[i], cx, cy, cz);
    const Shift3 sx = shifts(cx, box.ncell[0], box.prd[0]);
    const Shift3 sy = shifts(cy, box.ncell[1], box.prd[1]);
    const Shift3 sz = shifts(cz, box.ncell[2], box.prd[2]);
      const double gix = gs[3 * i], giy = gs[3 * i + 1], giz = gs[3 * i + 2];
    const int num = numneigh[i];
    double hx = 0.0, hy = 0.0, hz = 0.0;
    for (int k = 0; k < num; k++) {
      const unsigned e = (unsigned)nlist[md_slab(k, i, stride)];
      const int j = md_entry_j(e);
      double dx, dy, dz, rsq;
      int tt;
      pair_geom<MIXED>(T, i, e, x4, xq, sx, sy, sz, box.qs, box.qs_lo, dx, dy, dz, rsq, tt);
      if (rsq < T.cutsq[tt]) {
        const double wx = gix - gs[3 * j], wy = giy - gs[3 * j + 1], wz = giz - gs[3 * j + 2];
        double phi, phis, r14, r8;
        if (MIXED) {
          const float r2i = 1.0f / (float)rsq, r6i = r2i * r2i * r2i;
          const float l1 = (float)T.lj1[tt], l2 = (float)T.lj2[tt];
          phi = (double)((l1 * r6i - l2) * r6i * r2i);
          phis = (double)((4.0f * l2 - 7.0f * l1 * r6i) * r6i * r2i * r2i);
          r14 = (double)(r6i * r6i * r2i);
          r8 = (double)(r6i * r2i);
        } else {
          const double r2i = 1.0 / rsq, r6i = r2i * r2i * r2i;
          const double l1 = T.lj1[tt], l2 = T.lj2[tt];
          phi = (l1 * r6i - l2) * r6i * r2i;
          phis = (4.0 * l2 - 7.0 * l1 * r6i) * r6i * r2i * r2i;
          r14 = r6i * r6i * r2i;
          r8 = r6i * r2i;
        }
        const double dw = dx * wx + dy * wy + dz * wz;
        const double s = 2.0 * phis * dw;
        hx += phi * wx + s * dx;
        hy += phi * wy + s * dy;
        hz += phi * wz + s * dz;
        const double gd = gix * dx + giy * dy + giz * dz;
#pragma unroll
        for (int p = 0; p < kAdjNP; p++) {
          acc[2 * p] += p == tt ? gd * r14 : 0.0;
          acc[2 * p + 1] += p == tt ? -gd * r8 : 0.0;
        }
      }
    }
    const int o = orig[i];
    gx[3 * o] = hx;
    gx[3 * o + 1] = hy;
    gx[3 * o + 2] = hz;
  }
  block_partials_finish<2 * kAdjNP>(acc, red, partial, counter, gtab, false);
}

AdjTables make_tables(const b200_ctx *c, const double *lj1, const double *lj2,
                      const double *cutsq) {
  AdjTables T{};
  T.ntypes = c->ntypes;
  const int w = c->ntypes + 1;
  for (int a = 1; a <= c->ntypes; a++)
    for (int b = 1; b <= c->ntypes; b++) {
      const int p = (a - 1) * c->ntypes + (b - 1);
      T.lj1[p] = lj1[a * w + b];
      T.lj2[p] = lj2[a * w + b];
      T.cutsq[p] = cutsq[a * w + b];
    }
  return T;
}

}  // namespace

cudaError_t md_adj_forward(b200_ctx *c, const double *lj1, const double *lj2, const double *cutsq,
                           double *f) {
  const AdjTables T = make_tables(c, lj1, lj2, cutsq);
  const int grid = md_blocks(c->n, kAdjThreads);
  if (c->prec == B200_PREC_MIXED)
    k_adj_forward<true><<<grid, kAdjThreads, 0, c->stream>>>(c->n, c->stride, T, c->box, c->x4,
                                                             c->xq, c->cell, c->nlist,
                                                             c->numneigh, c->orig, f);
  else
    k_adj_forward<false><<<grid, kAdjThreads, 0, c->stream>>>(c->n, c->stride, T, c->box, c->x4,
                                                              c->xq, c->cell, c->nlist,
                                                              c->numneigh, c->orig, f);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_adj_backward(b200_ctx *c, const double *lj1, const double *lj2,
                            const double *cutsq, const double *g, double *gx, double *gs,
                            double *gtab) {
  const AdjTables T = make_tables(c, lj1, lj2, cutsq);
  const int grid = md_blocks(c->n, kAdjThreads);
  k_adj_gather<<<md_blocks(c->n, 256), 256, 0, c->stream>>>(c->n, c->orig, g, gs);
  if (c->prec == B200_PREC_MIXED)
    k_adj_backward<true><<<grid, kAdjThreads, 0, c->stream>>>(
        c->n, c->stride, T, c->box, c->x4, c->xq, c->cell, c->nlist, c->numneigh, c->orig, gs, gx,
        c->partial, c->counter, gtab);
  else
    k_adj_backward<false><<<grid, kAdjThreads, 0, c->stream>>>(
        c->n, c->stride, T, c->box, c->x4, c->xq, c->cell, c->nlist, c->numneigh, c->orig, gs, gx,
        c->partial, c->counter, gtab);
  c->launches += 2;
  return cudaGetLastError();
}

// caller-order device positions -> the context's sorted FP64 positions
// (types kept, image flags restarted); the next build wraps and re-sorts
__global__ void k_adj_positions(int n, const int *__restrict__ orig, const double *__restrict__ x,
                                double4 *__restrict__ x4, int *__restrict__ image) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = orig[i];
  const double4 p = x4[i];
  x4[i] = make_double4(x[3 * o], x[3 * o + 1], x[3 * o + 2], p.w);
  image[i] = md_img_pack(0, 0, 0);
}

cudaError_t md_adj_positions(b200_ctx *c, const double *x) {
  k_adj_positions<<<md_blocks(c->n, 256), 256, 0, c->stream>>>(c->n, c->orig, x, c->x4, c->image);
  c->launches++;
  return cudaGetLastError();
}
