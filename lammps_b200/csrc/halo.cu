// halo.cu -- per-step forward communication of ghost positions for a
// spatially decomposed box.
//
// A rank's context holds its own atoms and, as ghosts, copies of the atoms of
// other ranks that lie within the ghost depth of its brick, all in the one
// periodic box.  Between rebuilds the ghost set is fixed and each step only
// refreshes ghost positions from their owners, as CommBrick::forward_comm
// does with AtomVecAtomic::pack_comm / unpack_comm
// (src/comm_brick.cpp:444-511, src/atom_vec_atomic.cpp:105-217).  The atoms
// are addressed by caller index (upload order); `where` maps a caller index
// to the atom's current slot in the cell-sorted order.  A ghost is a copy of
// the owner's coordinates, not a periodic image: the builder forms the images.
#include "md_state.h"

namespace {

// new coordinates of sorted slot k, with the fixed-point copy (mixed form)
// formed as the integrator forms it
__device__ __forceinline__ void set_position(int k, double x, double y, double z,
                                             double4 *__restrict__ x4, int4 *__restrict__ xq,
                                             const BoxGeom &box) {
  double4 p = x4[k];
  p.x = x;
  p.y = y;
  p.z = z;
  x4[k] = p;
  if (xq) xq[k] = md_xq(p, box);
}

__global__ void k_where(int n, const int *__restrict__ orig, int *__restrict__ where) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) where[orig[k]] = k;
}

__global__ void k_halo_pack(int m, int n, const int *__restrict__ idx,
                            const int *__restrict__ where, const double4 *__restrict__ x4,
                            double *__restrict__ buf, int *__restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int j = idx[i];
  if (j < 0 || j >= n) {
    atomicExch(&status[ST_HALO_BAD], 1);
    return;
  }
  const double4 p = x4[where[j]];
  buf[3 * (size_t)i] = p.x;
  buf[3 * (size_t)i + 1] = p.y;
  buf[3 * (size_t)i + 2] = p.z;
}

// `ghost` (caller order) is given when the context has ghosts marked: an index
// that names an owned atom is refused, since writing it would overwrite a
// position that the rank's own integrator carries forward
__global__ void k_halo_unpack(int m, int n, const int *__restrict__ idx,
                              const int *__restrict__ where, const int *__restrict__ ghost,
                              const double *__restrict__ buf, double4 *__restrict__ x4,
                              int4 *__restrict__ xq, BoxGeom box, int *__restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int j = idx[i];
  if (j < 0 || j >= n) {
    atomicExch(&status[ST_HALO_BAD], 1);
    return;
  }
  if (ghost && ghost[j] == 0) {
    atomicExch(&status[ST_HALO_BAD], 2);
    return;
  }
  const int k = where[j];
  set_position(k, buf[3 * (size_t)i], buf[3 * (size_t)i + 1], buf[3 * (size_t)i + 2], x4, xq,
               box);
}

// every atom: x of sorted slot k = x[orig[k]] (caller order); a batched
// context forms each atom's fixed-point copy in its own replica's box
__global__ void k_positions(int n, const int *__restrict__ orig, const double *__restrict__ x,
                            double4 *__restrict__ x4, int4 *__restrict__ xq, BoxGeom box,
                            Reps reps, int batch) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const size_t o = (size_t)orig[k];
  set_position(k, x[3 * o], x[3 * o + 1], x[3 * o + 2], x4, xq,
               batch ? reps.box[reps.rep_of_atom[k]] : box);
}

}  // namespace

cudaError_t md_where(b200_ctx *c) {
  if (c->n < 1) return cudaSuccess;
  k_where<<<md_blocks(c->n, 256), 256, 0, c->stream>>>(c->n, c->orig, c->where);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_halo_pack(b200_ctx *c, int m, const int *idx, double *buf) {
  if (m < 1) return cudaSuccess;
  k_halo_pack<<<md_blocks(m, 256), 256, 0, c->stream>>>(m, c->n, idx, c->where, c->x4, buf,
                                                        c->status);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_halo_unpack(b200_ctx *c, int m, const int *idx, const double *buf) {
  if (m < 1) return cudaSuccess;
  k_halo_unpack<<<md_blocks(m, 256), 256, 0, c->stream>>>(
      m, c->n, idx, c->where, c->ghosts_on ? c->ghost : nullptr, buf, c->x4,
      c->prec == B200_PREC_MIXED ? c->xq : nullptr, c->box, c->status);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_set_positions(b200_ctx *c, const double *x) {
  if (c->n < 1) return cudaSuccess;
  k_positions<<<md_blocks(c->n, 256), 256, 0, c->stream>>>(
      c->n, c->orig, x, c->x4, c->prec == B200_PREC_MIXED ? c->xq : nullptr, c->box, c->reps(),
      c->nrep > 0);
  c->launches++;
  return cudaGetLastError();
}
