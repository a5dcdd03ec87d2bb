// replica.cu -- per-replica reductions of a batched context.
//
// A batched context advances many independent periodic boxes with the same
// kernels as one box (every kernel looks up its atom's or tile's replica).
// The global energy/virial sums of those kernels mix the replicas, so the
// thermo quantities of each replica -- ComputeTemp's sum m v^2, ComputePE's
// eng_vdwl and ComputePressure's virial (src/compute_temp.cpp:59-89,
// src/compute_pe.cpp:71-100, src/compute_pressure.cpp:177-207) -- are
// reduced here, one CTA per replica, in a fixed order.
#include "md_state.h"

namespace {

constexpr int kRepThreads = 256;

// rows[9 r + ...] = {natoms, sum m v^2, eng_vdwl, virial[0..5]} of replica r.
// The atoms of replica r are the sorted indices [atom_start[r],
// atom_start[r+1]) and, in the caller's order, the same index range.
__global__ void __launch_bounds__(kRepThreads)
    k_rep_rows(const int *__restrict__ atom_start, int stride, const double *__restrict__ mass,
               const double4 *__restrict__ x4, const double *__restrict__ v,
               const double *__restrict__ eatom, const double *__restrict__ vatom,
               double *__restrict__ rows) {
  __shared__ double red[8 * (kRepThreads / 32)];
  const int r = blockIdx.x;
  const int a0 = atom_start[r], a1 = atom_start[r + 1];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = a0 + threadIdx.x; k < a1; k += blockDim.x) {
    const double m = mass[(int)x4[k].w];
    const double vx = v[k], vy = v[stride + k], vz = v[2 * stride + k];
    acc[0] += (vx * vx + vy * vy + vz * vz) * m;
    acc[1] += eatom[k];
#pragma unroll
    for (int q = 0; q < 6; q++) acc[2 + q] += vatom[6 * (size_t)k + q];
  }
  block_sum<8>(acc, red);
  if (threadIdx.x == 0) {
    double *row = rows + 9 * (size_t)r;
    row[0] = (double)(a1 - a0);
#pragma unroll
    for (int q = 0; q < 8; q++) row[1 + q] = acc[q];
  }
}

}  // namespace

cudaError_t md_rep_rows(b200_ctx *c, const int *d_start, const double *eatom, const double *vatom,
                        double *rows) {
  // d_start: device copy of the replica atom ranges (nrep + 1 ints)
  k_rep_rows<<<c->nrep, kRepThreads, 0, c->stream>>>(d_start, c->stride, c->mass_dev, c->x4, c->v,
                                                     eatom, vatom, rows);
  c->launches++;
  return cudaGetLastError();
}
