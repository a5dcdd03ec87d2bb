// md_common.cuh -- shared device definitions of the B200 MD engine.
//
// Device-resident layout of one box (all arrays in cell-sorted order):
//   x4[i]      double4 (x, y, z, type)       -- FP64 positions, gathered per pair
//   v[3][n]    double SoA                     -- velocities
//   f[3][n]    double SoA                     -- forces (owner-summed; no ghosts)
//   xr[i]      float4 (cell-relative x,y,z, type bits) -- mixed precision only
//   cell[i]    packed cell coordinates cx | cy<<10 | cz<<20 of the last build
//   nlist      ELL neighbor list, entry k of atom i at nlist[k*stride + i]:
//              bits 0..26 = neighbor atom index, bits 27..31 = cell offset
//              code (dcx+1) + 3(dcy+1) + 9(dcz+1) of the neighbor's cell.
// Periodic images are never stored: a neighbor in a wrapped cell is the owner
// atom plus the box shift implied by the offset code, so the reference's
// ghost atoms, forward_comm and reverse_comm disappear.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define MD_MAXTYPES 8
#define MD_JBITS 27
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
  ST_COUNT = 16
};

struct BoxGeom {
  double lo[3], hi[3], prd[3];
  double cinv[3];    // cells per unit length: ncell/prd
  double cs[3];      // cell edge prd/ncell
  int ncell[3];
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

// image flags packed as LAMMPS imageint: 10 bits per dimension, offset 512
// (src/lmptype.h IMGMAX/IMGBITS)
#define MD_IMGMAX 512
#define MD_IMGMASK 1023
__host__ __device__ inline int md_img_pack(int ix, int iy, int iz) {
  return ((iz + MD_IMGMAX) & MD_IMGMASK) << 20 | ((iy + MD_IMGMAX) & MD_IMGMASK) << 10 |
         ((ix + MD_IMGMAX) & MD_IMGMASK);
}

// FP64 helpers that keep a*b+c rounded twice, as the reference's x86-64
// build computes them; used wherever a comparison must be bit-exact.
__device__ __forceinline__ double dsq3(double a, double b, double c) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
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
    // threads of the last block sum one component each, in block order
    for (int k = threadIdx.x; k < NV; k += blockDim.x) {
      double s = 0.0;
      for (unsigned int b = 0; b < gridDim.x; b++) s += __ldcg(&partial[(size_t)b * NV + k]);
      out[k] = accumulate ? out[k] + s : s;
    }
    if (threadIdx.x == 0) *counter = 0u;
  }
}
