// api.cu -- the C ABI of libb200md (include/b200md.h): context lifetime,
// settings, atom transfer, setup, the per-step entry points and the
// graph-captured Verlet loop.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <algorithm>
#include <vector>

#include <atomic>
#include <chrono>

#include "md_state.h"

namespace {

int set_err(b200_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_err(c, B200_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                               \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
  }
  if (count == 0) return cudaSuccess;
  return cudaMalloc((void **)p, count * sizeof(T));
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void invalidate_graphs(b200_ctx *c) {
  for (int k = 0; k < MD_NGRAPHS; k++) {
    if (c->step_exec[k]) cudaGraphExecDestroy(c->step_exec[k]);
    if (c->step_graph[k]) cudaGraphDestroy(c->step_graph[k]);
    c->step_exec[k] = nullptr;
    c->step_graph[k] = nullptr;
    c->ev_nodes[k].clear();
    c->step_kernels[k] = 0;
  }
  c->graph_valid = false;
}

// true for device (or managed) memory, false for host memory of any kind
bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The context's transfer staging: `parts` byte counts laid out one after
// another (256-byte aligned) in one device buffer that only grows.  Growing
// synchronizes the stream first, since queued copies may still use it.
int xfer_parts(b200_ctx *c, int nparts, const size_t *bytes, char **ptrs) {
  size_t total = 0;
  for (int k = 0; k < nparts; k++) total += (bytes[k] + 255) & ~(size_t)255;
  if (total > c->xfer_bytes) {
    CK(cudaStreamSynchronize(c->stream));
    if (c->xfer) cudaFree(c->xfer);
    c->xfer = nullptr;
    c->xfer_bytes = 0;
    CK(cudaMalloc((void **)&c->xfer, total));
    c->xfer_bytes = total;
  }
  size_t off = 0;
  for (int k = 0; k < nparts; k++) {
    ptrs[k] = bytes[k] ? c->xfer + off : nullptr;
    off += (bytes[k] + 255) & ~(size_t)255;
  }
  return B200_OK;
}

// ---- kernels local to the ABI ------------------------------------------------

__global__ void k_upload(int n, int stride, int ntypes, const double *__restrict__ x,
                         const double *__restrict__ v, const int *__restrict__ type,
                         double4 *__restrict__ x4, double *__restrict__ vd,
                         int *__restrict__ orig, int *__restrict__ image,
                         int *__restrict__ cell, int *__restrict__ status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int t = type[i];
  if (t < 1 || t > ntypes) {  // recorded for the host (one offending index), kept in range
    atomicCAS(&status[ST_BADTYPE], 0, i + 1);
    t = 1;
  }
  x4[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], (double)t);
  vd[i] = v ? v[3 * i] : 0.0;
  vd[stride + i] = v ? v[3 * i + 1] : 0.0;
  vd[2 * stride + i] = v ? v[3 * i + 2] : 0.0;
  orig[i] = i;
  image[i] = md_img_pack(0, 0, 0);
  cell[i] = 0;
}

__global__ void k_unsort(int n, int stride, const int *__restrict__ orig,
                         const double4 *__restrict__ x4, const double *__restrict__ v,
                         const double *__restrict__ f, const int *__restrict__ image,
                         double *__restrict__ xo, double *__restrict__ vo, double *__restrict__ fo,
                         int *__restrict__ io) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = orig[i];
  if (xo) {
    const double4 p = x4[i];
    xo[3 * o] = p.x;
    xo[3 * o + 1] = p.y;
    xo[3 * o + 2] = p.z;
  }
  if (vo) {
    vo[3 * o] = v[i];
    vo[3 * o + 1] = v[stride + i];
    vo[3 * o + 2] = v[2 * stride + i];
  }
  if (fo) {
    fo[3 * o] = f[i];
    fo[3 * o + 1] = f[stride + i];
    fo[3 * o + 2] = f[2 * stride + i];
  }
  if (io) {
    const int img = image[i];
    io[3 * o] = (img & MD_IMGMASK) - MD_IMGMAX;
    io[3 * o + 1] = ((img >> 10) & MD_IMGMASK) - MD_IMGMAX;
    io[3 * o + 2] = ((img >> 20) & MD_IMGMASK) - MD_IMGMAX;
  }
}

// per-atom columns of m atoms (caller indices idx, or 0..m-1) in row-major
// order: x y z | vx vy vz | fx fy fz | ix iy iz, the requested groups only
__global__ void k_gather_cols(int m, int n, int stride, int fields, int ncols,
                              const int *__restrict__ idx, const int *__restrict__ where,
                              const double4 *__restrict__ x4, const double *__restrict__ v,
                              const double *__restrict__ f, const int *__restrict__ image,
                              double *__restrict__ out, int *__restrict__ status) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int o = idx ? idx[r] : r;
  if (o < 0 || o >= n) {  // recorded for the host; the row is left as it is
    atomicExch(&status[ST_HALO_BAD], 1);
    return;
  }
  const int k = where[o];
  double *row = out + (size_t)r * ncols;
  int c = 0;
  if (fields & B200_FIELD_X) {
    const double4 p = x4[k];
    row[c++] = p.x;
    row[c++] = p.y;
    row[c++] = p.z;
  }
  if (fields & B200_FIELD_V) {
    row[c++] = v[k];
    row[c++] = v[stride + k];
    row[c++] = v[2 * stride + k];
  }
  if (fields & B200_FIELD_F) {
    row[c++] = f[k];
    row[c++] = f[stride + k];
    row[c++] = f[2 * stride + k];
  }
  if (fields & B200_FIELD_IMAGE) {
    const int img = image[k];
    row[c++] = (double)((img & MD_IMGMASK) - MD_IMGMAX);
    row[c++] = (double)(((img >> 10) & MD_IMGMASK) - MD_IMGMAX);
    row[c++] = (double)(((img >> 20) & MD_IMGMASK) - MD_IMGMAX);
  }
}

__global__ void k_unsort_scalar(int n, const int *__restrict__ orig, const double *__restrict__ a,
                                double *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[orig[i]] = a[i];
}

__global__ void k_full_total(int n, const int *__restrict__ numneigh,
                             unsigned long long *__restrict__ total) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v = i < n ? (unsigned long long)numneigh[i] : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(total, v);
}

// ---- host helpers --------------------------------------------------------------

int check_ready(b200_ctx *c) {
  if (!c->box_set) return set_err(c, B200_ERR_STATE, "box not set");
  if (!c->have_atoms) return set_err(c, B200_ERR_STATE, "no atoms uploaded");
  if (c->pstyle == B200_PAIR_NONE) return set_err(c, B200_ERR_STATE, "no pair style set");
  if (!c->mass_set) return set_err(c, B200_ERR_STATE, "masses not set");
  if (c->nrep && c->rep_atom_start[c->nrep] != c->n)
    return set_err(c, B200_ERR_STATE, "replica atom counts sum to %d, %d atoms uploaded",
                   c->rep_atom_start[c->nrep], c->n);
  if (c->nrep && c->pstyle != B200_PAIR_LJ_CUT)
    return set_err(c, B200_ERR_STATE, "replicas run pair_style lj/cut");
  return B200_OK;
}

// The cell grid of one periodic box for neighbor cutoff cutneighmax: cells
// at least cutneighmax wide, one periodic image per side
// (CommBrick::setup, src/comm_brick.cpp:128-170).
// Fixed-point scale of the mixed form's coordinates (md_xq): 2^32 units per
// box edge.  A listed pair must sit at its minimum image, so the mixed form
// needs every edge longer than twice the list cutoff.
int box_fixed_point(b200_ctx *c, BoxGeom &b) {
  for (int d = 0; d < 3; d++) {
    if (c->prec == B200_PREC_MIXED && !(b.prd[d] > 2.0 * c->cutneighmax))
      return set_err(c, B200_ERR_BOX,
                     "mixed precision needs box edges longer than twice the list cutoff: edge "
                     "%g in dim %d, list cutoff %g",
                     b.prd[d], d, c->cutneighmax);
    b.qinv[d] = 4294967296.0 / b.prd[d];
    const double u = b.prd[d] / 4294967296.0;  // exact: a power-of-two scale
    b.qs[d] = (float)u;
    b.qs_lo[d] = (float)(u - (double)b.qs[d]);
  }
  const double q2 = 1.0 / ((b.prd[0] / 4294967296.0) * (b.prd[0] / 4294967296.0));
  b.q2inv = (float)q2;
  b.q2inv_lo = (float)(q2 - (double)b.q2inv);
  b.qiso = b.prd[0] == b.prd[1] && b.prd[1] == b.prd[2];
  return B200_OK;
}

int box_cells(b200_ctx *c, BoxGeom &b, long long *ncells) {
  *ncells = 1;
  for (int d = 0; d < 3; d++) {
    int maxneed = (int)(c->cutneighmax * 1 / b.prd[d]) + 1;
    if (maxneed != 1)
      return set_err(c, B200_ERR_BOX, "box edge %g in dim %d is not larger than the ghost cutoff %g",
                     b.prd[d], d, c->cutneighmax);
    int nc = (int)(b.prd[d] / c->cutneighmax);
    if (nc < 1) nc = 1;
    if (nc > MD_MAX_CELLS_DIM - 1) nc = MD_MAX_CELLS_DIM - 1;
    b.ncell[d] = nc;
    b.cs[d] = b.prd[d] / nc;
    b.cinv[d] = nc / b.prd[d];
    *ncells *= nc;
  }
  return box_fixed_point(c, b);
}

// Cell grids, cell and builder-tile offsets of every replica, and their
// device copies (b200_set_replicas).
int init_replica_cells(b200_ctx *c) {
  const int R = c->nrep;
  c->rep_cell_base.assign(R, 0);
  c->rep_tile_base.assign(R + 1, 0);
  long long cells = 0, tiles = 0;
  for (int r = 0; r < R; r++) {
    long long nc = 0;
    int rc = box_cells(c, c->rep_box[r], &nc);
    if (rc) return set_err(c, rc, "replica %d: %s", r, c->err.c_str());
    c->rep_cell_base[r] = (int)cells;
    c->rep_tile_base[r] = (int)tiles;
    cells += nc;
    const BoxGeom &b = c->rep_box[r];
    tiles += (long long)((b.ncell[0] + MD_TILE_CELLS - 1) / MD_TILE_CELLS) * b.ncell[1] * b.ncell[2];
  }
  c->rep_tile_base[R] = (int)tiles;
  if (cells > (long long)4096 * 4096 - 1 || tiles > 0x7fffffffLL)
    return set_err(c, B200_ERR_ARG, "too many cells (%lld)", cells);
  if ((int)cells != c->ncells || (int)tiles != c->ntiles) invalidate_graphs(c);
  c->ncells = (int)cells;
  c->ntiles = (int)tiles;
  c->box = c->rep_box[0];
  std::vector<int> tile_rep(tiles), rep_of_atom(c->n);
  for (int r = 0; r < R; r++) {
    for (int t = c->rep_tile_base[r]; t < c->rep_tile_base[r + 1]; t++) tile_rep[t] = r;
    for (int i = c->rep_atom_start[r]; i < c->rep_atom_start[r + 1]; i++) rep_of_atom[i] = r;
  }
  if (c->rep_dev_r < R) {
    CK(dalloc(&c->d_rep_box, (size_t)R));
    CK(dalloc(&c->d_rep_cell_base, (size_t)R));
    CK(dalloc(&c->d_rep_tile_base, (size_t)R + 1));
    c->rep_dev_r = R;
    invalidate_graphs(c);
  }
  if (c->rep_dev_tiles < (int)tiles) {
    CK(dalloc(&c->d_tile_rep, (size_t)tiles));
    c->rep_dev_tiles = (int)tiles;
    invalidate_graphs(c);
  }
  if (c->rep_dev_n < c->n) {
    CK(dalloc(&c->d_rep_of_atom, (size_t)c->n));
    c->rep_dev_n = c->n;
    invalidate_graphs(c);
  }
  CK(cudaMemcpy(c->d_rep_box, c->rep_box.data(), R * sizeof(BoxGeom), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_rep_cell_base, c->rep_cell_base.data(), R * sizeof(int),
                cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_rep_tile_base, c->rep_tile_base.data(), (R + 1) * sizeof(int),
                cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_tile_rep, tile_rep.data(), tiles * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_rep_of_atom, rep_of_atom.data(), c->n * sizeof(int),
                cudaMemcpyHostToDevice));
  return B200_OK;
}

// Neighbor::init cutoffs (src/neighbor.cpp:255-279) and the cell grid
int init_cutoffs_and_cells(b200_ctx *c) {
  const int ntp1 = c->ntypes + 1;
  double cutsq[TABSZ];
  for (int i = 0; i < TABSZ; i++) cutsq[i] = 0.0;
  if (c->pstyle == B200_PAIR_LJ_CUT) {
    for (int i = 1; i <= c->ntypes; i++)
      for (int j = 1; j <= c->ntypes; j++) cutsq[i * ntp1 + j] = c->lj.cutsq[i * ntp1 + j];
  } else {
    for (int i = 1; i <= c->ntypes; i++)
      for (int j = 1; j <= c->ntypes; j++) cutsq[i * ntp1 + j] = c->eam.cutmax * c->eam.cutmax;
  }
  c->cutneighmax = 0.0;
  c->cutforce_max = 0.0;
  for (int i = 1; i <= c->ntypes; i++)
    for (int j = 1; j <= c->ntypes; j++) {
      const double cutoff = std::sqrt(cutsq[i * ntp1 + j]);
      const double delta = cutoff > 0.0 ? c->skin : 0.0;
      const double cut = cutoff + delta;
      c->cutneighsq[i * ntp1 + j] = cut * cut;
      if (cut > c->cutneighmax) c->cutneighmax = cut;
      if (cutoff > c->cutforce_max) c->cutforce_max = cutoff;
    }
  if (!(c->cutneighmax > 0.0)) return set_err(c, B200_ERR_ARG, "zero neighbor cutoff");
  if (c->nrep) return init_replica_cells(c);
  long long ncells = 1;
  for (int d = 0; d < 3; d++) {
    // CommBrick::setup needs one periodic image per side: cutghost < prd
    int maxneed = (int)(c->cutneighmax * 1 / c->box.prd[d]) + 1;
    if (maxneed != 1)
      return set_err(c, B200_ERR_BOX, "box edge %g in dim %d is not larger than the ghost cutoff %g",
                     c->box.prd[d], d, c->cutneighmax);
    int nc = (int)(c->box.prd[d] / c->cutneighmax);
    if (nc < 1) nc = 1;
    if (nc > MD_MAX_CELLS_DIM - 1) nc = MD_MAX_CELLS_DIM - 1;
    c->box.ncell[d] = nc;
    c->box.cs[d] = c->box.prd[d] / nc;
    c->box.cinv[d] = nc / c->box.prd[d];
    ncells *= nc;
  }
  if (int rc = box_fixed_point(c, c->box)) return rc;
  if (ncells > (long long)4096 * 4096 - 1)
    return set_err(c, B200_ERR_ARG, "too many cells (%lld)", ncells);
  if ((int)ncells != c->ncells) invalidate_graphs(c);  // scan launch shape changes
  c->ncells = (int)ncells;
  return B200_OK;
}

int upload_tables(b200_ctx *c) {
  const int ntp1 = c->ntypes + 1;
  std::vector<double> tab(TAB_COUNT * TABSZ, 0.0);
  for (int k = 0; k < ntp1 * ntp1; k++) {
    tab[TAB_CUTNEIGHSQ * TABSZ + k] = c->cutneighsq[k];
    tab[TAB_CUTSQ * TABSZ + k] = c->lj.cutsq[k];
    tab[TAB_LJ1 * TABSZ + k] = c->lj.lj1[k];
    tab[TAB_LJ2 * TABSZ + k] = c->lj.lj2[k];
    tab[TAB_LJ3 * TABSZ + k] = c->lj.lj3[k];
    tab[TAB_LJ4 * TABSZ + k] = c->lj.lj4[k];
    tab[TAB_OFFSET * TABSZ + k] = c->lj.offset[k];
  }
  std::vector<int> maps((MD_MAXTYPES + 1) + 2 * TABSZ, 0);
  for (int k = 0; k < ntp1; k++) maps[k] = c->eam.type2frho[k];
  for (int k = 0; k < ntp1 * ntp1; k++) {
    maps[(MD_MAXTYPES + 1) + k] = c->eam.type2rhor[k];
    maps[(MD_MAXTYPES + 1) + TABSZ + k] = c->eam.type2z2r[k];
  }
  if (!c->tables_dev) {
    size_t bytes = TAB_COUNT * TABSZ * sizeof(double) + maps.size() * sizeof(int);
    CK(cudaMalloc((void **)&c->tables_dev, bytes));
    c->cutneighsq_dev = c->tables_dev + TAB_CUTNEIGHSQ * TABSZ;
  }
  CK(cudaMemcpyAsync(c->tables_dev, tab.data(), tab.size() * sizeof(double),
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->tables_dev + TAB_COUNT * TABSZ, maps.data(), maps.size() * sizeof(int),
                     cudaMemcpyHostToDevice, c->stream));
  std::vector<double> m(MD_MAXTYPES + 1, 1.0);
  for (int t = 1; t <= c->ntypes; t++) m[t] = c->mass[t];
  if (!c->mass_dev) CK(cudaMalloc((void **)&c->mass_dev, (MD_MAXTYPES + 1) * sizeof(double)));
  CK(cudaMemcpyAsync(c->mass_dev, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

int alloc_cells(b200_ctx *c) {
  if (c->ncells + 1 > c->ncell_alloc) {
    invalidate_graphs(c);
    int m = c->ncells + 1;
    CK(dalloc(&c->cell_count, (size_t)m));
    // zero once here: each build's scatter zeroes the counts for the next
    CK(cudaMemsetAsync(c->cell_count, 0, (size_t)m * sizeof(int), c->stream));
    CK(dalloc(&c->cell_start, (size_t)m));
    CK(dalloc(&c->scan_tmp, (size_t)4096 + 1));
    c->ncell_alloc = m;
  }
  return B200_OK;
}

int alloc_list(b200_ctx *c, int capacity) {
  capacity = (capacity + 3) & ~3;  // whole int4 slabs
  long long need = (long long)capacity * c->stride;
  if (capacity != c->capacity) invalidate_graphs(c);  // capacity is a kernel argument
  if (need > c->nlist_alloc) {
    invalidate_graphs(c);
    CK(dalloc(&c->nlist, (size_t)need));
    c->nlist_alloc = need;
  }
  c->capacity = capacity;
  return B200_OK;
}

int default_capacity(const b200_ctx *c) {
  double dens = c->n / (c->box.prd[0] * c->box.prd[1] * c->box.prd[2]);
  for (int r = 0; r < c->nrep; r++) {
    const BoxGeom &b = c->rep_box[r];
    const double d = c->rep_natoms[r] / (b.prd[0] * b.prd[1] * b.prd[2]);
    dens = r == 0 ? d : (d > dens ? d : dens);
  }
  const double pi = 3.14159265358979323846;
  const double expect = 4.0 / 3.0 * pi * c->cutneighmax * c->cutneighmax * c->cutneighmax * dens;
  int cap = (int)(2.0 * expect + 64.0);
  cap = (cap + 7) & ~7;
  return cap;
}

// Small device-to-host reads (status words, energy and virial sums, step
// counters) go through mapped page-locked memory, written by a one-warp
// kernel on the context's stream.  A copy engine would queue them behind a
// bulk transfer in flight in the same direction (b200_download_atoms_async),
// and the host would wait for that transfer to end.
constexpr int kBounceBytes = 4096;

__global__ void k_small_read(const int *__restrict__ src, int *__restrict__ dst, int nwords) {
  for (int k = threadIdx.x; k < nwords; k += blockDim.x) dst[k] = src[k];
  __threadfence_system();
}

// `bytes` (a multiple of 4, at most kBounceBytes) from device `dev` into host
// `host`, after the work already queued on the stream
int small_read(b200_ctx *c, void *host, const void *dev, size_t bytes) {
  if (bytes % 4 != 0 || bytes > (size_t)kBounceBytes)
    return set_err(c, B200_ERR_ARG, "small read of %zu bytes", bytes);
  k_small_read<<<1, 32, 0, c->stream>>>(reinterpret_cast<const int *>(dev), c->bounce_dev,
                                        (int)(bytes / 4));
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(host, c->bounce_host, bytes);
  return B200_OK;
}

int read_status(b200_ctx *c) { return small_read(c, c->status_host, c->status, ST_COUNT * sizeof(int)); }

int status_errors(b200_ctx *c) {
  if (c->status_host[ST_LOST])
    return set_err(c, B200_ERR_LOST_ATOMS,
                   "Lost atoms: a coordinate is not finite or moved beyond one box length");
  if (c->status_host[ST_OVERFLOW])
    return set_err(c, B200_ERR_NEIGH_OVERFLOW,
                   "Neighbor list overflow, boost neigh_modify one (need %d, have %d)",
                   c->status_host[ST_MAXNEIGH], c->capacity);
  return B200_OK;
}

int pair_compute_dev(b200_ctx *c, bool ev, bool atom, double *eatom, double *vatom) {
  cudaError_t e;
  if (c->pstyle == B200_PAIR_LJ_CUT) e = md_lj_compute(c, ev, atom, eatom, vatom);
  else e = md_eam_compute(c, ev, atom, eatom, vatom);
  if (e != cudaSuccess) return set_err(c, B200_ERR_CUDA, "pair kernel: %s", cudaGetErrorString(e));
  return B200_OK;
}

// rebuild with overflow recovery (host-synchronous; setup and b200_neigh_build)
int rebuild_sync(b200_ctx *c) {
  for (int attempt = 0; attempt < 3; attempt++) {
    CK(cudaMemsetAsync(c->status + ST_MAXNEIGH, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->status + ST_OVERFLOW, 0, sizeof(int), c->stream));
    CK(md_rebuild(c, nullptr));
    int rc = read_status(c);
    if (rc) return rc;
    if (c->status_host[ST_LOST]) return status_errors(c);
    if (md_stage_feedback(c, c->status_host[ST_MAXSTAGE])) invalidate_graphs(c);
    if (!c->status_host[ST_OVERFLOW]) return B200_OK;
    if (c->one_user > 0) return status_errors(c);
    int need = c->status_host[ST_MAXNEIGH];
    int cap = ((int)(need * 1.2) + 32 + 7) & ~7;
    rc = alloc_list(c, cap);
    if (rc) return rc;
    invalidate_graphs(c);
    // the atoms are already in cell order; the repeat rebuild keeps them
  }
  return set_err(c, B200_ERR_NEIGH_OVERFLOW, "Neighbor list overflow, boost neigh_modify one");
}

// Launch-shape search of a box that steps through the one-launch step kernel
// (md_lj_step / md_eam_step): the step kernel itself is timed, for 1, 2, 4
// and 8 threads per atom, since its best shape can differ from the two-kernel
// pair pass's (at 32,000 LJ atoms, mixed: 2 and 4 tie for the pair pass, 4 is
// 6 % faster for the step).  The steps run with a zero timestep, so
// positions and velocities do not change; the status words, the decision
// count and the mailbox that the steps advance are put back afterwards.  It
// runs at setup and, once, between two steps of the first run.
int autotune_step(b200_ctx *c) {
  int status_save[ST_COUNT], dcount_save = 0;
  int rc0 = small_read(c, status_save, c->status, sizeof(status_save));
  if (!rc0) rc0 = small_read(c, &dcount_save, c->dec_count, sizeof(int));
  if (rc0) return rc0;
  const int mail_save[2] = {c->mail_host[0], c->mail_host[1]};
  const int parity_save = c->pos_parity;
  const bool lj = c->pstyle == B200_PAIR_LJ_CUT;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int cand[4] = {1, 2, 4, 8};
  float tmin[4] = {1e30f, 1e30f, 1e30f, 1e30f};
  auto step = [&]() -> cudaError_t {
    cudaError_t e = lj ? md_lj_step(c, 0.0, 0.0, false) : md_eam_step(c, 0.0, 0.0, false);
    md_swap_positions(c);
    return e;
  };
  // one timed block of `reps` steps at the current shape
  auto block = [&](int reps, float &ms) -> cudaError_t {
    cudaError_t e = cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = step();
    if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    return e;
  };
  // Warm-up (clocks up, caches filled) at one thread per atom, which also
  // sizes the timed blocks: about 2 ms of steps, 5 to 40 of them (a block
  // of five 40-microsecond steps at 32,000 atoms picked different shapes
  // from one context to the next).
  int rc = B200_OK;
  c->tpa = 1;
  float ms = 0.f;
  cudaError_t e = block(10, ms);
  int reps = 5;
  if (e == cudaSuccess) reps = std::max(5, std::min(40, (int)ceilf(20.0f / std::max(ms, 1e-3f))));
  else rc = set_err(c, B200_ERR_CUDA, "launch-shape search: %s", cudaGetErrorString(e));
  for (int round = 0; round < 3 && !rc; round++)
    for (int k = 0; k < 4 && !rc; k++) {
      c->tpa = cand[k];
      e = step();
      if (e == cudaSuccess) e = block(reps, ms);
      if (e != cudaSuccess) rc = set_err(c, B200_ERR_CUDA, "launch-shape search: %s",
                                         cudaGetErrorString(e));
      else if (ms < tmin[k]) tmin[k] = ms;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // back to the buffer the search started from (after a zero-timestep step
  // both buffers hold the same positions)
  if (c->pos_parity != parity_save) md_swap_positions(c);
  CK(cudaMemcpyAsync(c->status, status_save, sizeof(status_save), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(c->dec_count, &dcount_save, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->mail_host[0] = mail_save[0];
  c->mail_host[1] = mail_save[1];
  if (rc) return rc;
  float best = 1e30f;
  int best_tpa = 1;
  for (int k = 0; k < 4; k++)
    if (tmin[k] < best * 0.97f) {
      best = tmin[k];
      best_tpa = cand[k];
    }
  c->tpa = best_tpa;
  c->tuned = true;
  return B200_OK;
}

// a single box of lj/cut (equal edges in the mixed form) or eam steps
// through the one-launch step kernel
static bool step_form(const b200_ctx *c) {
  return c->nrep == 0 && !c->ghosts_on &&
         ((c->pstyle == B200_PAIR_LJ_CUT && (c->prec != B200_PREC_MIXED || md_q_iso(c))) ||
          c->pstyle == B200_PAIR_EAM);
}

int autotune(b200_ctx *c) {
  if (step_form(c)) return autotune_step(c);
  // Launch-shape search: time the force pass for each threads-per-atom
  // value and keep the fastest (ties to fewer threads per atom).  Each
  // candidate is timed in three rounds of five passes, the rounds
  // interleaved across the candidates, and its fastest round counts: at a
  // few microseconds per pass a single short timing picked different shapes
  // from run to run.
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int cand[6] = {1, 2, 4, 8, 16, 32};
  float tmin[6] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
  for (int round = 0; round < 3; round++)
    for (int k = 0; k < 6; k++) {
      c->tpa = cand[k];
      int rc = pair_compute_dev(c, false, false, nullptr, nullptr);
      if (rc) return rc;
      CK(cudaEventRecord(e0, c->stream));
      for (int r = 0; r < 5; r++) {
        rc = pair_compute_dev(c, false, false, nullptr, nullptr);
        if (rc) return rc;
      }
      CK(cudaEventRecord(e1, c->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < tmin[k]) tmin[k] = ms;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  float best = 1e30f;
  int best_tpa = 1;
  for (int k = 0; k < 6; k++)
    if (tmin[k] < best * 0.97f) {
      best = tmin[k];
      best_tpa = cand[k];
    }
  c->tpa = best_tpa;
  c->tuned = true;
  return B200_OK;
}

int count_kernels(b200_ctx *c, cudaGraph_t g, int *kernels, std::vector<cudaGraphNode_t> *events) {
  size_t nn = 0;
  CK(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  CK(cudaGraphGetNodes(g, nodes.data(), &nn));
  *kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) (*kernels)++;
    if (events && t == cudaGraphNodeTypeEventRecord) events->push_back(nd);
  }
  return B200_OK;
}

// A step (Verlet::run body, src/verlet.cpp:223-308) is three pieces:
//   PRE     fix nve initial half-step + the rebuild decision
//   REBUILD wrap, cell sort, neighbor list (only on rebuild steps)
//   POST    pair forces, fix nve final half-step (+ kinetic energy and thermo
//           row on output steps)
// The host launches REBUILD exactly when the reference's Neighbor::decide
// would rebuild: it mirrors the `ago` counter, so with `check no` the
// schedule needs no device read-back, and with `check yes` it reads the
// device's distance test only on the steps where a rebuild is possible.
// Each piece is a captured CUDA graph (or, with graphs off, its kernels
// launched one by one).  With timing on, events mark the phase boundaries:
// PRE holds phases 0-1, POST phases 2-5; their events are swapped per
// launch so every step's phases can be read back.
enum {
  PIECE_PRE = 0,
  PIECE_REBUILD = 1,
  PIECE_POST_OUT = 2,
  PIECE_POST = 3,
  PIECE_FUSED_OUT = 4,  // POST_OUT + the next step's initial half-step and decision
  PIECE_FUSED = 5       // POST + the same
};

cudaError_t record(b200_ctx *c, cudaEvent_t ev) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(c->stream, &st);
  return st == cudaStreamCaptureStatusActive
             ? cudaEventRecordWithFlags(ev, c->stream, cudaEventRecordExternal)
             : cudaEventRecord(ev, c->stream);
}

// launch the kernels of one piece; ev (optional) are the piece's events
cudaError_t launch_piece(b200_ctx *c, int kind, double dtv, double dtf, cudaEvent_t *ev) {
  cudaError_t e = cudaSuccess;
  if (kind == PIECE_PRE) {
    if (ev) e = record(c, ev[0]);
    if (e == cudaSuccess) e = md_nve_initial(c, dtv, dtf);
    if (e == cudaSuccess) e = md_decide(c);
    if (e == cudaSuccess && ev) e = record(c, ev[1]);
  } else if (kind == PIECE_REBUILD) {
    e = md_rebuild(c, nullptr);
  } else {
    const bool out = kind == PIECE_POST_OUT || kind == PIECE_FUSED_OUT;
    const bool fused = kind == PIECE_FUSED_OUT || kind == PIECE_FUSED;
    if (fused && md_lj_step_ok(c)) {
      // lj/cut: this step's forces, final half-step and thermo row and the
      // next step's initial half-step and decision in one launch (the caller
      // swaps the position buffers after it)
      return md_lj_step(c, dtv, dtf, out);
    }
    if (fused && md_eam_step_ok(c)) return md_eam_step(c, dtv, dtf, out);  // the same for eam
    if (ev) e = record(c, ev[0]);
    if (kind == PIECE_FUSED && c->rep_onelaunch && c->nrep && c->pstyle == B200_PAIR_LJ_CUT) {
      // replicas: this step's forces, final half-step and the next step's
      // initial half-step and decision in one cluster launch
      return md_rep_step(c, dtv, dtf);
    }
    if (e == cudaSuccess) {
      if (c->pstyle == B200_PAIR_LJ_CUT) {
        e = md_lj_compute(c, out, false, nullptr, nullptr);
        if (e == cudaSuccess && ev) e = record(c, ev[1]);
      } else {
        e = md_eam_compute(c, out, false, nullptr, nullptr, ev ? ev[1] : nullptr);
      }
    }
    if (e == cudaSuccess && ev) e = record(c, ev[2]);
    // the fused half-steps also record the thermo row and make the next
    // step's rebuild decision (in their last block)
    if (e == cudaSuccess) e = fused ? md_nve_fused(c, dtv, dtf, out) : md_nve_final(c, dtf, out);
    if (e == cudaSuccess && out && !fused) e = md_record_row(c);
    if (e == cudaSuccess && ev) e = record(c, ev[3]);
  }
  return e;
}

// Step form of a replica batch: device time per step of the graph path's
// fused piece (pair kernel + fused half-steps) and of the one-launch step for
// each cluster size, block size and threads per atom, keeping the fastest.
// The steps are timed with a zero timestep, so positions and velocities do
// not change; the step counters, rebuild schedule and decision mailbox that
// the steps advance are put back afterwards.
int tune_replica_step(b200_ctx *c) {
  const bool lj = c->pstyle == B200_PAIR_LJ_CUT;
  c->rep_onelaunch = false;
  c->rep_tune_ms[0] = c->rep_tune_ms[1] = 0.0;
  if (!c->nrep || !lj || c->rep_mode == 1) return B200_OK;
  int status_save[ST_COUNT], dcount_save = 0;
  int rc0 = small_read(c, status_save, c->status, sizeof(status_save));
  if (!rc0) rc0 = small_read(c, &dcount_save, c->dec_count, sizeof(int));
  if (rc0) return rc0;
  const int mail_save[2] = {c->mail_host[0], c->mail_host[1]};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int steps = 16;
  auto time_steps = [&](bool one, float *ms) -> int {
    for (int r = 0; r < steps + 2; r++) {
      if (r == 2) CK(cudaEventRecord(e0, c->stream));
      CK(one ? md_rep_step(c, 0.0, 0.0) : launch_piece(c, PIECE_FUSED, 0.0, 0.0, nullptr));
    }
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    *ms /= steps;
    return B200_OK;
  };
  float graph_ms = 1e30f;
  int rc = B200_OK;
  if (c->rep_mode == 0) rc = time_steps(false, &graph_ms);
  float best = 1e30f;
  int bcs = 0, bblock = 0, btpa = 0;
  const int cs_c[3] = {1, 2, 4}, bl_c[2] = {256, 512}, tp_c[3] = {1, 2, 4};
  for (int a = 0; a < 3 && !rc; a++)
    for (int b = 0; b < 2 && !rc; b++)
      for (int t = 0; t < 3 && !rc; t++) {
        if ((c->rep_fix_cs > 0 && cs_c[a] != c->rep_fix_cs) ||
            (c->rep_fix_block > 0 && bl_c[b] != c->rep_fix_block) ||
            (c->rep_fix_tpa > 0 && tp_c[t] != c->rep_fix_tpa))
          continue;
        rc = md_rep_plan(c, cs_c[a], bl_c[b], tp_c[t]);
        float ms = 0.f;
        if (!rc) rc = time_steps(true, &ms);
        if (!rc && ms < best) {
          best = ms;
          bcs = cs_c[a];
          bblock = bl_c[b];
          btpa = tp_c[t];
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc && bcs) rc = md_rep_plan(c, bcs, bblock, btpa);
  CK(cudaMemcpyAsync(c->status, status_save, sizeof(status_save), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(c->dec_count, &dcount_save, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->mail_host[0] = mail_save[0];
  c->mail_host[1] = mail_save[1];
  if (rc) return rc;
  c->rep_tune_ms[0] = graph_ms < 1e29f ? graph_ms : 0.0;
  c->rep_tune_ms[1] = best < 1e29f ? best : 0.0;
  c->rep_onelaunch = bcs > 0 && (c->rep_mode == 2 || best < graph_ms);
  c->rep_tuned = true;
  invalidate_graphs(c);
  return B200_OK;
}

// captures piece `kind` for the current position buffers, in graph slot
// kind + MD_NPIECES * pos_parity
int capture_piece(b200_ctx *c, int kind, double dtv, double dtf) {
  const int slot = kind + MD_NPIECES * c->pos_parity;
  const bool tm = c->timing && kind != PIECE_REBUILD;
  const long long launches0 = c->launches;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = launch_piece(c, kind, dtv, dtf, tm ? c->ph_event : nullptr);
  cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
  c->launches = launches0;
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return set_err(c, B200_ERR_CUDA, "graph capture: %s / %s", cudaGetErrorString(e),
                   cudaGetErrorString(e2));
  }
  int kernels = 0;
  c->ev_nodes[slot].clear();
  int rc = count_kernels(c, g, &kernels, &c->ev_nodes[slot]);
  if (rc) {
    cudaGraphDestroy(g);
    return rc;
  }
  const size_t want = !tm ? 0 : (kind == PIECE_PRE ? 2 : 4);
  if (c->ev_nodes[slot].size() != want) {
    cudaGraphDestroy(g);
    return set_err(c, B200_ERR_CUDA, "graph capture: expected %zu event nodes, found %zu", want,
                   c->ev_nodes[slot].size());
  }
  e = cudaGraphInstantiate(&c->step_exec[slot], g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return set_err(c, B200_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  c->step_graph[slot] = g;
  c->step_kernels[slot] = kernels;
  return B200_OK;
}

// The rebuild decision of the last piece launched: wait until the device's
// decision count in the mailbox reaches the host's, then read the flag.  If
// that takes longer than 0.2 s, read the status word after a stream
// synchronize instead (which also reports a CUDA error) and take the
// device's count as the host's.
int wait_decision(b200_ctx *c, bool *rebuild) {
  volatile int *m = c->mail_host;
  const int want = (int)c->decisions;
  const auto t0 = std::chrono::steady_clock::now();
  for (unsigned it = 1;; it++) {
    if (m[1] == want) {
      std::atomic_thread_fence(std::memory_order_acquire);
      *rebuild = m[0] != 0;
      return B200_OK;
    }
    if ((it & 4095u) == 0u &&
        std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(200))
      break;
  }
  int dc = 0;
  int rc1 = small_read(c, &c->status_host[ST_REBUILD], c->status + ST_REBUILD, sizeof(int));
  if (!rc1) rc1 = small_read(c, &dc, c->dec_count, sizeof(int));
  if (rc1) return rc1;
  c->decisions = (unsigned int)dc;
  *rebuild = c->status_host[ST_REBUILD] != 0;
  return B200_OK;
}

// run one piece: graph replay, or the kernels themselves with graphs off.  A
// fused piece that ran md_lj_step leaves the new positions in the other
// buffer, which becomes current.
int run_piece(b200_ctx *c, int kind, double dtv, double dtf, cudaEvent_t *ev) {
  const bool swap = (kind == PIECE_FUSED || kind == PIECE_FUSED_OUT) && md_step_ok(c);
  if (!c->use_graphs) {
    CK(launch_piece(c, kind, dtv, dtf, ev));
  } else {
    const int slot = kind + MD_NPIECES * c->pos_parity;
    if (ev)
      for (size_t k = 0; k < c->ev_nodes[slot].size(); k++)
        CK(cudaGraphExecEventRecordNodeSetEvent(c->step_exec[slot], c->ev_nodes[slot][k], ev[k]));
    CK(cudaGraphLaunch(c->step_exec[slot], c->stream));
    c->launches += c->step_kernels[slot];
  }
  if (swap) md_swap_positions(c);
  return B200_OK;
}

int ensure_graphs(b200_ctx *c, double dtv, double dtf, double ftm2v) {
  if (!c->use_graphs) return B200_OK;
  if (c->graph_valid) return B200_OK;
  // with md_lj_step the position buffers alternate from step to step: every
  // piece is captured for both (the pointer swap is host state only)
  const int sets = md_step_ok(c) ? 2 : 1;
  for (int set = 0; set < sets; set++) {
    if (set) md_swap_positions(c);
    for (int kind = 0; kind < MD_NPIECES; kind++) {
      // the fused pieces are not used with phase timers on (their events
      // would mix two steps)
      if (c->timing && (kind == PIECE_FUSED || kind == PIECE_FUSED_OUT)) continue;
      int rc = capture_piece(c, kind, dtv, dtf);
      if (rc) {
        if (set) md_swap_positions(c);
        return rc;
      }
    }
    if (set) md_swap_positions(c);
  }
  c->graph_valid = true;
  c->graph_dt = dtv;
  c->graph_ftm2v = ftm2v;
  c->graph_tpa = c->tpa;
  c->graph_timing = c->timing;
  return B200_OK;
}

// Larger neighbor-list capacity.  keep = true copies the current entries
// (entry k of atom i sits at k*stride + i, so the old list is a prefix).
int grow_list(b200_ctx *c, int capacity, bool keep) {
  capacity = (capacity + 3) & ~3;  // whole int4 slabs
  if (capacity <= c->capacity) return B200_OK;
  long long need = (long long)capacity * c->stride;
  if (need > c->nlist_alloc) {
    int *nl = nullptr;
    CK(cudaMalloc((void **)&nl, (size_t)need * sizeof(int)));
    if (keep && c->nlist)
      CK(cudaMemcpyAsync(nl, c->nlist, (size_t)c->capacity * c->stride * sizeof(int),
                         cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->nlist) cudaFree(c->nlist);
    c->nlist = nl;
    c->nlist_alloc = need;
  }
  c->capacity = capacity;
  invalidate_graphs(c);
  return B200_OK;
}

// Save (save = true) or restore the per-atom state and status words that a
// run chunk changes.
int snapshot(b200_ctx *c, bool save) {
  const size_t s = (size_t)c->stride;
  if (c->snap_alloc < c->stride) {
    CK(dalloc(&c->snap_x4, s));
    CK(dalloc(&c->snap_xhold, s));
    CK(dalloc(&c->snap_v, 3 * s));
    CK(dalloc(&c->snap_f, 3 * s));
    CK(dalloc(&c->snap_orig, s));
    CK(dalloc(&c->snap_image, s));
    CK(dalloc(&c->snap_cell, s));
    CK(dalloc(&c->snap_xq, s));
    if (!c->snap_status) CK(cudaMalloc((void **)&c->snap_status, ST_COUNT * sizeof(int)));
    c->snap_alloc = c->stride;
  }
  auto cp = [&](void *a, void *b, size_t bytes) -> cudaError_t {
    return save ? cudaMemcpyAsync(b, a, bytes, cudaMemcpyDeviceToDevice, c->stream)
                : cudaMemcpyAsync(a, b, bytes, cudaMemcpyDeviceToDevice, c->stream);
  };
  const size_t n = (size_t)c->n;
  CK(cp(c->x4, c->snap_x4, n * sizeof(double4)));
  CK(cp(c->v, c->snap_v, 3 * s * sizeof(double)));
  CK(cp(c->f, c->snap_f, 3 * s * sizeof(double)));
  CK(cp(c->orig, c->snap_orig, n * sizeof(int)));
  CK(cp(c->image, c->snap_image, n * sizeof(int)));
  CK(cp(c->cell, c->snap_cell, n * sizeof(int)));
  if (c->check) CK(cp(c->xhold, c->snap_xhold, n * sizeof(double4)));
  if (c->prec == B200_PREC_MIXED) CK(cp(c->xq, c->snap_xq, n * sizeof(int4)));
  CK(cp(c->status, c->snap_status, ST_COUNT * sizeof(int)));
  if (!save) CK(md_where(c));
  return B200_OK;
}

int ensure_events(b200_ctx *c, size_t count) {
  for (int k = 0; k <= MD_NPHASE; k++)
    if (!c->ph_event[k]) CK(cudaEventCreate(&c->ph_event[k]));
  while (c->ev_pool.size() < count) {
    cudaEvent_t ev;
    CK(cudaEventCreate(&ev));
    c->ev_pool.push_back(ev);
  }
  return B200_OK;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================

extern "C" {

int b200_abi_version(void) { return B200MD_ABI_VERSION; }

int b200_create(int device, int precision, b200_ctx **out) {
  if (!out) return B200_ERR_ARG;
  *out = nullptr;
  if (precision != B200_PREC_FP64 && precision != B200_PREC_MIXED) return B200_ERR_ARG;
  b200_ctx *c = new (std::nothrow) b200_ctx();
  if (!c) return B200_ERR_NOMEM;
  c->device = device;
  c->prec = precision;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->s_aux, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->status, ST_COUNT * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->status, 0, ST_COUNT * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->status_host, ST_COUNT * sizeof(int));
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&c->mail_host, 4 * sizeof(int), cudaHostAllocMapped);
  if (e == cudaSuccess) {
    c->mail_host[0] = c->mail_host[1] = 0;
    e = cudaHostGetDevicePointer((void **)&c->mail_dev, c->mail_host, 0);
  }
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&c->bounce_host, kBounceBytes, cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&c->bounce_dev, c->bounce_host, 0);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->dec_count, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->dec_count, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->ev, 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(c->ev, 0, 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->counter, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(c->counter, 0, sizeof(unsigned int));
  if (e != cudaSuccess) {
    // report through a context so the caller can read the message
    c->err = std::string("b200_create: ") + cudaGetErrorString(e);
    *out = c;
    return B200_ERR_CUDA;
  }
  *out = c;
  return B200_OK;
}

int b200_destroy(b200_ctx *c) {
  if (!c) return B200_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->s_h2d) {
    cudaStreamSynchronize(c->s_h2d);
    cudaStreamSynchronize(c->s_d2h);
    for (auto *s : {&c->in_slot[0], &c->in_slot[1], &c->out_slot[0], &c->out_slot[1]}) {
      if (s->buf) cudaFree(s->buf);
      if (s->ready) cudaEventDestroy(s->ready);
      if (s->done) cudaEventDestroy(s->done);
    }
    cudaStreamDestroy(c->s_h2d);
    cudaStreamDestroy(c->s_d2h);
  }
  invalidate_graphs(c);
  dfree(c->x4); dfree(c->x4b); dfree(c->v); dfree(c->vb); dfree(c->f);
  dfree(c->orig); dfree(c->origb); dfree(c->image); dfree(c->imageb); dfree(c->cell);
  dfree(c->where); dfree(c->ghost);
  dfree(c->xq); dfree(c->xqb); dfree(c->xhold); dfree(c->xfer); dfree(c->rho); dfree(c->fp); dfree(c->fpf); dfree(c->mass_dev);
  dfree(c->eam_eatom); dfree(c->d_rep_grp_first); dfree(c->d_rep_ranges);
  dfree(c->cell_count); dfree(c->cell_start); dfree(c->scan_tmp);
  dfree(c->slot); dfree(c->perm); dfree(c->cell_tmp);
  dfree(c->nlist); dfree(c->numneigh); dfree(c->partial); dfree(c->counter); dfree(c->ev);
  dfree(c->adj_gs); dfree(c->adj_gtab);
  dfree(c->d_rep_box); dfree(c->d_rep_of_atom); dfree(c->d_rep_cell_base); dfree(c->d_tile_rep);
  dfree(c->d_rep_tile_base); 
  dfree(c->status); dfree(c->rows); dfree(c->tables_dev);
  dfree(c->snap_x4); dfree(c->snap_xhold); dfree(c->snap_v); dfree(c->snap_f);
  dfree(c->snap_orig); dfree(c->snap_image); dfree(c->snap_cell); dfree(c->snap_xq);
  dfree(c->snap_status);
  dfree(c->eam.frho); dfree(c->eam.rhor); dfree(c->eam.z2r);
  dfree(c->eam.frho_f); dfree(c->eam.rhor_f); dfree(c->eam.z2r_f); dfree(c->eam.fz_f);
  for (auto &ev : c->ph_event)
    if (ev) cudaEventDestroy(ev);
  for (auto ev : c->ev_pool) cudaEventDestroy(ev);
  if (c->status_host) cudaFreeHost(c->status_host);
  if (c->mail_host) cudaFreeHost(c->mail_host);
  if (c->bounce_host) cudaFreeHost(c->bounce_host);
  dfree(c->dec_count);
  if (c->s_aux) cudaStreamDestroy(c->s_aux);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return B200_OK;
}

const char *b200_last_error(const b200_ctx *c) { return c ? c->err.c_str() : "null context"; }

long long b200_bytes(const b200_ctx *c) {
  if (!c) return 0;
  long long s = (long long)c->stride;
  long long b = s * (2 * 32 + 2 * 24 + 24 + 5 * 4 + 16 + 32 + 16 + 4) + c->nlist_alloc * 4 +
                (long long)c->ncell_alloc * 8;
  return b;
}

int b200_set_box(b200_ctx *c, const double lo[3], const double hi[3]) {
  if (!c || !lo || !hi) return B200_ERR_ARG;
  for (int d = 0; d < 3; d++) {
    if (!(hi[d] > lo[d]) || !std::isfinite(lo[d]) || !std::isfinite(hi[d]))
      return set_err(c, B200_ERR_ARG, "Illegal box: hi <= lo in dim %d", d);
    c->box.lo[d] = lo[d];
    c->box.hi[d] = hi[d];
    c->box.prd[d] = hi[d] - lo[d];  // Domain::set_global_box
  }
  c->box_set = true;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_set_neighbor(b200_ctx *c, double skin, int every, int delay, int check, int one) {
  if (!c) return B200_ERR_ARG;
  if (!(skin >= 0.0) || every <= 0 || delay < 0)
    return set_err(c, B200_ERR_ARG, "Illegal neighbor command");
  c->skin = skin;
  c->every = every;
  c->delay = delay;
  c->check = check ? 1 : 0;
  if (one != c->one_user) c->capacity = 0;  // re-size the list at the next setup
  c->one_user = one;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_set_mass(b200_ctx *c, int ntypes, const double *mass) {
  if (!c || !mass || ntypes < 1 || ntypes > MD_MAXTYPES)
    return set_err(c, B200_ERR_ARG, "Illegal mass: ntypes must be 1..%d", MD_MAXTYPES);
  for (int t = 1; t <= ntypes; t++) {
    if (!(mass[t] > 0.0)) return set_err(c, B200_ERR_ARG, "Invalid mass value for type %d", t);
    c->mass[t] = mass[t];
  }
  if (c->ntypes && c->ntypes != ntypes)
    return set_err(c, B200_ERR_ARG, "mass table has %d types, pair style %d", ntypes, c->ntypes);
  c->ntypes = ntypes;
  c->mass_set = true;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_set_lj(b200_ctx *c, int ntypes, const double *cutsq, const double *lj1, const double *lj2,
                const double *lj3, const double *lj4, const double *offset) {
  if (!c || ntypes < 1 || ntypes > MD_MAXTYPES || !cutsq || !lj1 || !lj2 || !lj3 || !lj4 || !offset)
    return set_err(c, B200_ERR_ARG, "Illegal lj/cut tables");
  if (c->ntypes && c->ntypes != ntypes)
    return set_err(c, B200_ERR_ARG, "lj/cut tables have %d types, masses %d", ntypes, c->ntypes);
  const int ntp1 = ntypes + 1;
  for (int i = 0; i < ntp1 * ntp1; i++) {
    c->lj.cutsq[i] = cutsq[i];
    c->lj.lj1[i] = lj1[i];
    c->lj.lj2[i] = lj2[i];
    c->lj.lj3[i] = lj3[i];
    c->lj.lj4[i] = lj4[i];
    c->lj.offset[i] = offset[i];
  }
  c->ntypes = ntypes;
  c->pstyle = B200_PAIR_LJ_CUT;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_set_eam(b200_ctx *c, int ntypes, int nrho, double drho, int nr, double dr, double rhomax,
                 double cutmax, int nfrho, const double *frho_spline, int nrhor,
                 const double *rhor_spline, int nz2r, const double *z2r_spline,
                 const int *type2frho, const int *type2rhor, const int *type2z2r) {
  if (!c || ntypes < 1 || ntypes > MD_MAXTYPES || nrho < 3 || nr < 3 || !(drho > 0) || !(dr > 0) ||
      nfrho < 1 || nrhor < 1 || nz2r < 1 || !frho_spline || !rhor_spline || !z2r_spline ||
      !type2frho || !type2rhor || !type2z2r || !(cutmax > 0))
    return set_err(c, B200_ERR_ARG, "Illegal eam tables");
  if (c->ntypes && c->ntypes != ntypes)
    return set_err(c, B200_ERR_ARG, "eam tables have %d types, masses %d", ntypes, c->ntypes);
  const int ntp1 = ntypes + 1;
  for (int i = 1; i <= ntypes; i++) {
    if (type2frho[i] < 0 || type2frho[i] >= nfrho)
      return set_err(c, B200_ERR_ARG, "type2frho out of range");
    for (int j = 1; j <= ntypes; j++) {
      if (type2rhor[i * ntp1 + j] < 0 || type2rhor[i * ntp1 + j] >= nrhor ||
          type2z2r[i * ntp1 + j] < 0 || type2z2r[i * ntp1 + j] >= nz2r)
        return set_err(c, B200_ERR_ARG, "type2rhor/type2z2r out of range");
    }
  }
  EAMDev &E = c->eam;
  E.nrho = nrho;
  E.nr = nr;
  E.drho = drho;
  E.dr = dr;
  E.rdr = 1.0 / dr;      // PairEAM::array2spline (src/MANYBODY/pair_eam.cpp:700-701)
  E.rdrho = 1.0 / drho;
  E.rhomax = rhomax;
  E.cutmax = cutmax;
  E.cutforcesq = cutmax * cutmax;  // PairEAM::init_one (:423)
  E.nfrho = nfrho;
  E.nrhor = nrhor;
  E.nz2r = nz2r;
  for (int i = 0; i < ntp1; i++) E.type2frho[i] = i == 0 ? 0 : type2frho[i];
  for (int i = 0; i < ntp1 * ntp1; i++) {
    E.type2rhor[i] = (i / ntp1 == 0 || i % ntp1 == 0) ? 0 : type2rhor[i];
    E.type2z2r[i] = (i / ntp1 == 0 || i % ntp1 == 0) ? 0 : type2z2r[i];
  }
  E.rhor_sym = true;
  for (int i = 1; i < ntp1; i++)
    for (int j = 1; j < ntp1; j++)
      if (E.type2rhor[i * ntp1 + j] != E.type2rhor[j * ntp1 + i]) E.rhor_sym = false;
  // repack [table][knot][7] -> [table][knot][8]; FP32 copies reordered
  // [c3 c4 c5 c6 | c0 c1 c2 0] for one-float4 value / derivative loads
  // FP64 rows: embedding [c0..c6 -]; density and pair (reorder) as the FP32
  // rows, [c3 c4 c5 c6 | c0 c1 c2 -]
  auto pack = [&](const double *src, int ntab, int nk, double **dd, float **df,
                  bool reorder) -> int {
    std::vector<double> d8((size_t)ntab * (nk + 1) * 8, 0.0);
    std::vector<float> f8((size_t)ntab * (nk + 1) * 8, 0.0f);
    for (size_t r = 0; r < (size_t)ntab * (nk + 1); r++) {
      if (reorder) {
        for (int k = 0; k < 4; k++) d8[r * 8 + k] = src[r * 7 + 3 + k];
        for (int k = 0; k < 3; k++) d8[r * 8 + 4 + k] = src[r * 7 + k];
      } else {
        for (int k = 0; k < 7; k++) d8[r * 8 + k] = src[r * 7 + k];
      }
      for (int k = 0; k < 4; k++) f8[r * 8 + k] = (float)src[r * 7 + 3 + k];
      for (int k = 0; k < 3; k++) f8[r * 8 + 4 + k] = (float)src[r * 7 + k];
    }
    CK(dalloc(dd, d8.size()));
    CK(dalloc(df, f8.size()));
    CK(cudaMemcpy(*dd, d8.data(), d8.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(*df, f8.data(), f8.size() * sizeof(float), cudaMemcpyHostToDevice));
    return B200_OK;
  };
  int rc = pack(frho_spline, nfrho, nrho, &E.frho, &E.frho_f, false);
  if (!rc) rc = pack(rhor_spline, nrhor, nr, &E.rhor, &E.rhor_f, true);
  if (!rc) rc = pack(z2r_spline, nz2r, nr, &E.z2r, &E.z2r_f, true);
  if (rc) return rc;
  if (ntypes == 1) {
    // one element: the z2 value and rho' coefficients of each knot in one
    // 32-byte record for the mixed force kernel
    const size_t ri = (size_t)E.type2rhor[ntp1 + 1], zi = (size_t)E.type2z2r[ntp1 + 1];
    std::vector<float> fz((size_t)(nr + 1) * 8, 0.0f);
    for (size_t m = 0; m <= (size_t)nr; m++) {
      for (int k = 0; k < 4; k++) fz[m * 8 + k] = (float)z2r_spline[(zi * (nr + 1) + m) * 7 + 3 + k];
      for (int k = 0; k < 3; k++) fz[m * 8 + 4 + k] = (float)rhor_spline[(ri * (nr + 1) + m) * 7 + k];
    }
    CK(dalloc(&E.fz_f, fz.size()));
    CK(cudaMemcpy(E.fz_f, fz.data(), fz.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  c->ntypes = ntypes;
  c->pstyle = B200_PAIR_EAM;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_upload_atoms(b200_ctx *c, int n, const double *x, const double *v, const int *type,
                      const int *tag) {
  (void)tag;
  if (!c || n < 1 || !x || !type) return set_err(c, B200_ERR_ARG, "Illegal atoms");
  if (n > MD_MAX_ATOMS) return set_err(c, B200_ERR_ARG, "too many atoms (%d > %d)", n, MD_MAX_ATOMS);
  if (c->ntypes < 1) return set_err(c, B200_ERR_STATE, "set masses or a pair style before atoms");
  CK(cudaSetDevice(c->device));
  // host arrays are checked here, device arrays by the upload kernel
  const bool dev_type = is_device_ptr(type);
  if (!dev_type)
    for (int i = 0; i < n; i++)
      if (type[i] < 1 || type[i] > c->ntypes)
        return set_err(c, B200_ERR_ARG, "Invalid atom type %d of atom %d", type[i], i);
  // step graphs bake the atom count and the buffer addresses
  if (n != c->n || n > c->nalloc) invalidate_graphs(c);
  if (n > c->nalloc) {
    // a count that grows again (a decomposed box's owned + ghost atoms
    // between rebuilds) gets 1/16 headroom, so it does not reallocate at
    // every small growth
    long long cap = c->nalloc > 0 ? (long long)n + n / 16 : n;
    if (cap > MD_MAX_ATOMS) cap = MD_MAX_ATOMS;
    const int stride = (int)((cap + 31) & ~31LL);
    CK(dalloc(&c->x4, stride));
    CK(dalloc(&c->x4b, stride));
    CK(dalloc(&c->v, 3 * (size_t)stride));
    CK(dalloc(&c->vb, 3 * (size_t)stride));
    CK(dalloc(&c->f, 3 * (size_t)stride));
    CK(dalloc(&c->orig, stride));
    CK(dalloc(&c->origb, stride));
    CK(dalloc(&c->image, stride));
    CK(dalloc(&c->imageb, stride));
    CK(dalloc(&c->cell, stride));
    CK(dalloc(&c->where, stride));
    CK(dalloc(&c->ghost, stride));
    CK(dalloc(&c->xq, stride));
    CK(dalloc(&c->xqb, stride));
    CK(dalloc(&c->xhold, stride));
    CK(dalloc(&c->rho, stride));
    CK(dalloc(&c->fp, stride));
    CK(dalloc(&c->fpf, stride));
    CK(dalloc(&c->slot, stride));
    CK(dalloc(&c->perm, stride));
    CK(dalloc(&c->cell_tmp, stride));
    CK(dalloc(&c->numneigh, stride));
    // one partial per block of the widest pair launch (32 threads per atom,
    // 128 threads per block)
    c->partial_blocks = stride / 4 + 64;
    CK(dalloc(&c->partial, (size_t)c->partial_blocks * 8));
    c->nalloc = (int)cap;
    c->stride = stride;
    c->nlist_alloc = 0;
    dfree(c->nlist);
  }
  c->n = n;
  CK(cudaMemsetAsync(c->f, 0, 3 * (size_t)c->stride * sizeof(double), c->stream));
  // host sources are copied into the staging buffer; device sources are read
  // by the upload kernel where they are
  const bool dev_x = is_device_ptr(x), dev_v = v && is_device_ptr(v);
  char *st[3];
  const size_t b3 = 3 * (size_t)n * sizeof(double);
  const size_t sb[3] = {dev_x ? 0 : b3, (v && !dev_v) ? b3 : 0,
                        dev_type ? 0 : (size_t)n * sizeof(int)};
  int rc = xfer_parts(c, 3, sb, st);
  if (rc) return rc;
  const double *dx = dev_x ? x : reinterpret_cast<const double *>(st[0]);
  const double *dv = (!v || dev_v) ? v : reinterpret_cast<const double *>(st[1]);
  const int *dt = dev_type ? type : reinterpret_cast<const int *>(st[2]);
  if (!dev_x) CK(cudaMemcpyAsync(st[0], x, b3, cudaMemcpyHostToDevice, c->stream));
  if (v && !dev_v) CK(cudaMemcpyAsync(st[1], v, b3, cudaMemcpyHostToDevice, c->stream));
  if (!dev_type)
    CK(cudaMemcpyAsync(st[2], type, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->status + ST_BADTYPE, 0, sizeof(int), c->stream));
  k_upload<<<md_blocks(n, 256), 256, 0, c->stream>>>(n, c->stride, c->ntypes, dx, dv, dt, c->x4,
                                                     c->v, c->orig, c->image, c->cell, c->status);
  c->launches++;
  CK(cudaGetLastError());
  CK(md_where(c));
  c->ghosts_on = false;  // a new atom set: the caller marks its ghosts again
  if (dev_type) {
    int rc2 = read_status(c);
    if (rc2) return rc2;
    if (c->status_host[ST_BADTYPE]) {
      c->have_atoms = false;
      return set_err(c, B200_ERR_ARG, "Invalid atom type of atom %d", c->status_host[ST_BADTYPE] - 1);
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  c->have_atoms = true;
  c->sorted_once = false;
  return B200_OK;
}

int b200_natoms(const b200_ctx *c) { return c ? c->n : 0; }

int b200_gather(b200_ctx *c, int fields, int m, const int *idx, double *out) {
  if (!c || !out || m < 0 || fields <= 0 ||
      (fields & ~(B200_FIELD_X | B200_FIELD_V | B200_FIELD_F | B200_FIELD_IMAGE)))
    return set_err(c, B200_ERR_ARG, "gather: bad fields or arguments");
  if (!c->have_atoms) return set_err(c, B200_ERR_STATE, "no atoms uploaded");
  if (!idx && m > c->n) return set_err(c, B200_ERR_ARG, "gather: %d rows of %d atoms", m, c->n);
  if (m == 0) return B200_OK;
  CK(cudaSetDevice(c->device));
  const int ncols = 3 * (((fields & B200_FIELD_X) != 0) + ((fields & B200_FIELD_V) != 0) +
                         ((fields & B200_FIELD_F) != 0) + ((fields & B200_FIELD_IMAGE) != 0));
  const size_t obytes = (size_t)m * ncols * sizeof(double);
  const bool dev_out = is_device_ptr(out);
  const bool dev_idx = idx && is_device_ptr(idx);
  char *st[2];
  const size_t sb[2] = {dev_out ? 0 : obytes, (idx && !dev_idx) ? (size_t)m * sizeof(int) : 0};
  int rc = xfer_parts(c, 2, sb, st);
  if (rc) return rc;
  double *dout = dev_out ? out : reinterpret_cast<double *>(st[0]);
  const int *didx = idx;
  if (idx && !dev_idx) {
    CK(cudaMemcpyAsync(st[1], idx, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    didx = reinterpret_cast<const int *>(st[1]);
  }
  CK(cudaMemsetAsync(c->status + ST_HALO_BAD, 0, sizeof(int), c->stream));
  k_gather_cols<<<md_blocks(m, 256), 256, 0, c->stream>>>(m, c->n, c->stride, fields, ncols, didx,
                                                          c->where, c->x4, c->v, c->f, c->image,
                                                          dout, c->status);
  c->launches++;
  CK(cudaGetLastError());
  if (!dev_out) CK(cudaMemcpyAsync(out, dout, obytes, cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  if (c->status_host[ST_HALO_BAD])
    return set_err(c, B200_ERR_ARG, "gather: an atom index is outside [0, %d)", c->n);
  return B200_OK;
}

int b200_update_positions(b200_ctx *c, const double *x) {
  if (!c || !x) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  const size_t bytes = 3 * (size_t)c->n * sizeof(double);
  const double *dx = x;
  if (!is_device_ptr(x)) {
    char *st[1];
    const size_t sb[1] = {bytes};
    int rc = xfer_parts(c, 1, sb, st);
    if (rc) return rc;
    CK(cudaMemcpyAsync(st[0], x, bytes, cudaMemcpyHostToDevice, c->stream));
    dx = reinterpret_cast<const double *>(st[0]);
  }
  CK(md_set_positions(c, dx));
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

int b200_download_atoms(b200_ctx *c, double *x, double *v, double *f, int *image) {
  if (!c) return B200_ERR_ARG;
  if (!c->have_atoms) return set_err(c, B200_ERR_STATE, "no atoms uploaded");
  CK(cudaSetDevice(c->device));
  const int n = c->n;
  char *st[4];
  const size_t d3 = 3 * (size_t)n * sizeof(double);
  const size_t sb[4] = {x ? d3 : 0, v ? d3 : 0, f ? d3 : 0, image ? 3 * (size_t)n * sizeof(int) : 0};
  int rc = xfer_parts(c, 4, sb, st);
  if (rc) return rc;
  double *dx = reinterpret_cast<double *>(st[0]), *dv = reinterpret_cast<double *>(st[1]);
  double *df = reinterpret_cast<double *>(st[2]);
  int *di = reinterpret_cast<int *>(st[3]);
  k_unsort<<<md_blocks(n, 256), 256, 0, c->stream>>>(n, c->stride, c->orig, c->x4, c->v, c->f,
                                                     c->image, dx, dv, df, di);
  c->launches++;
  CK(cudaGetLastError());
  // host or device destinations (unified addressing)
  if (x) CK(cudaMemcpyAsync(x, dx, 3 * (size_t)n * sizeof(double), cudaMemcpyDefault, c->stream));
  if (v) CK(cudaMemcpyAsync(v, dv, 3 * (size_t)n * sizeof(double), cudaMemcpyDefault, c->stream));
  if (f) CK(cudaMemcpyAsync(f, df, 3 * (size_t)n * sizeof(double), cudaMemcpyDefault, c->stream));
  if (image) CK(cudaMemcpyAsync(image, di, 3 * (size_t)n * sizeof(int), cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

// ---- overlapped transfers ----------------------------------------------------

// the copy streams and the slots' events, made on first use
static int xfer_streams(b200_ctx *c) {
  if (c->s_h2d) return B200_OK;
  CK(cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking));
  for (auto *s : {&c->in_slot[0], &c->in_slot[1], &c->out_slot[0], &c->out_slot[1]}) {
    CK(cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming));
  }
  return B200_OK;
}

// a slot's device buffer of at least `bytes` (the slot is idle when called)
static int slot_reserve(b200_ctx *c, b200_ctx::XferSlot &s, size_t bytes) {
  if (s.bytes >= bytes) return B200_OK;
  if (s.buf) CK(cudaFree(s.buf));
  s.buf = nullptr;
  s.bytes = 0;
  CK(cudaMalloc((void **)&s.buf, bytes));
  s.bytes = bytes;
  return B200_OK;
}

static size_t part_bytes(size_t b) { return (b + 255) & ~(size_t)255; }

int b200_stage_atoms(b200_ctx *c, int n, const double *x, const double *v, const int *type) {
  if (!c || n < 1 || !x || !type) return set_err(c, B200_ERR_ARG, "stage: illegal atoms");
  if (n > MD_MAX_ATOMS) return set_err(c, B200_ERR_ARG, "too many atoms (%d > %d)", n, MD_MAX_ATOMS);
  if (c->in_count == 2) return set_err(c, B200_ERR_STATE, "stage: two atom sets are staged already");
  CK(cudaSetDevice(c->device));
  int rc = xfer_streams(c);
  if (rc) return rc;
  b200_ctx::XferSlot &s = c->in_slot[(c->in_head + c->in_count) % 2];
  const size_t b3 = 3 * (size_t)n * sizeof(double), bt = (size_t)n * sizeof(int);
  // a free slot: the set it held was taken by b200_set_staged_atoms, which
  // returns after the upload that read it
  rc = slot_reserve(c, s, 2 * part_bytes(b3) + part_bytes(bt));
  if (rc) return rc;
  CK(cudaMemcpyAsync(s.buf, x, b3, cudaMemcpyDefault, c->s_h2d));
  if (v) CK(cudaMemcpyAsync(s.buf + part_bytes(b3), v, b3, cudaMemcpyDefault, c->s_h2d));
  CK(cudaMemcpyAsync(s.buf + 2 * part_bytes(b3), type, bt, cudaMemcpyDefault, c->s_h2d));
  CK(cudaEventRecord(s.ready, c->s_h2d));
  s.n = n;
  s.has_v = v != nullptr;
  c->in_count++;
  return B200_OK;
}

int b200_set_staged_atoms(b200_ctx *c) {
  if (!c) return B200_ERR_ARG;
  if (c->in_count == 0) return set_err(c, B200_ERR_STATE, "no staged atom set");
  CK(cudaSetDevice(c->device));
  b200_ctx::XferSlot &s = c->in_slot[c->in_head];
  c->in_head = (c->in_head + 1) % 2;
  c->in_count--;
  // the upload waits for the set's copy on the device, then reads the slot
  // (device memory: the types are checked by the upload kernel)
  CK(cudaStreamWaitEvent(c->stream, s.ready, 0));
  const size_t b3 = part_bytes(3 * (size_t)s.n * sizeof(double));
  return b200_upload_atoms(c, s.n, reinterpret_cast<const double *>(s.buf),
                           s.has_v ? reinterpret_cast<const double *>(s.buf + b3) : nullptr,
                           reinterpret_cast<const int *>(s.buf + 2 * b3), nullptr);
}

int b200_download_atoms_async(b200_ctx *c, double *x, double *v, double *f, int *image) {
  if (!c) return B200_ERR_ARG;
  if (!c->have_atoms) return set_err(c, B200_ERR_STATE, "no atoms uploaded");
  CK(cudaSetDevice(c->device));
  int rc = xfer_streams(c);
  if (rc) return rc;
  const int n = c->n;
  b200_ctx::XferSlot &s = c->out_slot[c->out_next];
  c->out_next ^= 1;
  const size_t d3 = 3 * (size_t)n * sizeof(double), i3 = 3 * (size_t)n * sizeof(int);
  const size_t pb[4] = {x ? part_bytes(d3) : 0, v ? part_bytes(d3) : 0, f ? part_bytes(d3) : 0,
                        image ? part_bytes(i3) : 0};
  const size_t need = pb[0] + pb[1] + pb[2] + pb[3];
  if (s.used && s.bytes < need) CK(cudaEventSynchronize(s.done));  // before freeing it
  rc = slot_reserve(c, s, need);
  if (rc) return rc;
  // the slot's previous copy to the host ends before the slot is written
  if (s.used) CK(cudaStreamWaitEvent(c->stream, s.done, 0));
  char *p[4];
  size_t off = 0;
  for (int k = 0; k < 4; k++) {
    p[k] = pb[k] ? s.buf + off : nullptr;
    off += pb[k];
  }
  k_unsort<<<md_blocks(n, 256), 256, 0, c->stream>>>(
      n, c->stride, c->orig, c->x4, c->v, c->f, c->image, reinterpret_cast<double *>(p[0]),
      reinterpret_cast<double *>(p[1]), reinterpret_cast<double *>(p[2]),
      reinterpret_cast<int *>(p[3]));
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(s.ready, c->stream));
  CK(cudaStreamWaitEvent(c->s_d2h, s.ready, 0));
  if (x) CK(cudaMemcpyAsync(x, p[0], d3, cudaMemcpyDefault, c->s_d2h));
  if (v) CK(cudaMemcpyAsync(v, p[1], d3, cudaMemcpyDefault, c->s_d2h));
  if (f) CK(cudaMemcpyAsync(f, p[2], d3, cudaMemcpyDefault, c->s_d2h));
  if (image) CK(cudaMemcpyAsync(image, p[3], i3, cudaMemcpyDefault, c->s_d2h));
  CK(cudaEventRecord(s.done, c->s_d2h));
  s.used = true;
  return B200_OK;
}

int b200_wait_transfers(b200_ctx *c) {
  if (!c) return B200_ERR_ARG;
  if (!c->s_h2d) return B200_OK;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->s_h2d));
  CK(cudaStreamSynchronize(c->s_d2h));
  return B200_OK;
}

static int prepare(b200_ctx *c) {
  int rc = check_ready(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  rc = init_cutoffs_and_cells(c);
  if (!rc) rc = upload_tables(c);
  if (!rc) rc = alloc_cells(c);
  if (!rc && (c->capacity == 0 || c->one_user > 0 || !c->nlist)) {
    int cap = c->one_user > 0   ? c->one_user
              : c->one_user < 0 ? (c->capacity > 0 ? c->capacity : -c->one_user)
              : (c->capacity > 0 ? c->capacity : default_capacity(c));
    rc = alloc_list(c, cap);
  }
  return rc;
}

int b200_neigh_build(b200_ctx *c) {
  if (!c) return B200_ERR_ARG;
  int rc = prepare(c);
  if (rc) return rc;
  rc = rebuild_sync(c);
  if (rc) return rc;
  c->sorted_once = true;
  return B200_OK;
}

int b200_pair_compute(b200_ctx *c, int eflag, int vflag, double *eng, double virial[6],
                      double *eatom, double *vatom) {
  if (!c) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  // Integrate::ev_set flags: eflag 1 global, 2 per-atom; vflag 1|2 global, 4 per-atom
  const bool eg = (eflag & 1) != 0, ea = (eflag & 2) != 0;
  const bool vg = (vflag % 4) != 0, va = (vflag & 4) != 0;
  const bool ev = eg || ea || vg || va;
  const bool atom = ea || va;
  const int n = c->n;
  char *st[2];
  const size_t sb[2] = {(ea && eatom) ? (size_t)n * sizeof(double) : 0,
                        (va && vatom) ? 6 * (size_t)n * sizeof(double) : 0};
  int rc = xfer_parts(c, 2, sb, st);
  if (rc) return rc;
  double *de = reinterpret_cast<double *>(st[0]), *dv = reinterpret_cast<double *>(st[1]);
  if (de) CK(cudaMemsetAsync(de, 0, (size_t)n * sizeof(double), c->stream));
  rc = pair_compute_dev(c, ev, atom, de, dv);
  if (rc) return rc;
  double h[8];
  if (ev) CK(cudaMemcpyAsync(h, c->ev, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (de) CK(cudaMemcpyAsync(eatom, de, (size_t)n * sizeof(double), cudaMemcpyDefault, c->stream));
  if (dv) CK(cudaMemcpyAsync(vatom, dv, 6 * (size_t)n * sizeof(double), cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (ev) {
    if (eg && eng) *eng = h[0];
    if (vg && virial)
      for (int k = 0; k < 6; k++) virial[k] = h[1 + k];
  }
  return B200_OK;
}

// ---- EAM in two calls with the F'(rho) forward communication between them --

static int eam_split_check(b200_ctx *c) {
  if (!c) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  if (c->pstyle != B200_PAIR_EAM) return set_err(c, B200_ERR_STATE, "pair style is not eam");
  CK(cudaSetDevice(c->device));
  return B200_OK;
}

int b200_eam_density(b200_ctx *c, int eflag, int vflag) {
  int rc = eam_split_check(c);
  if (rc) return rc;
  const bool eg = (eflag & 1) != 0, ea = (eflag & 2) != 0;
  const bool vg = (vflag % 4) != 0, va = (vflag & 4) != 0;
  if (ea && c->eam_eatom_n < c->n) {
    dfree(c->eam_eatom);
    CK(dalloc(&c->eam_eatom, (size_t)c->nalloc));
    c->eam_eatom_n = c->nalloc;
  }
  CK(md_eam_compute(c, eg || ea || vg || va, ea || va, ea ? c->eam_eatom : nullptr, nullptr,
                    nullptr, EAM_DENSITY));
  CK(cudaStreamSynchronize(c->stream));
  c->eam_split_eflag = eflag;
  c->eam_split_vflag = vflag;
  return B200_OK;
}

static int eam_fp_call(b200_ctx *c, int m, const int *idx, double *buf, bool pack) {
  int rc = eam_split_check(c);
  if (rc) return rc;
  if (m < 0 || (m > 0 && (!idx || !buf))) return set_err(c, B200_ERR_ARG, "Illegal F' halo");
  if (m == 0) return B200_OK;
  CK(cudaMemsetAsync(c->status + ST_HALO_BAD, 0, sizeof(int), c->stream));
  CK(md_eam_fp_halo(c, m, idx, buf, pack));
  rc = read_status(c);
  if (rc) return rc;
  if (c->status_host[ST_HALO_BAD] == 2)
    return set_err(c, B200_ERR_ARG, "F' unpack: an index names an owned atom, not a ghost");
  if (c->status_host[ST_HALO_BAD])
    return set_err(c, B200_ERR_ARG, "F' %s: an atom index is outside [0, %d)",
                   pack ? "pack" : "unpack", c->n);
  return B200_OK;
}

int b200_eam_fp_pack(b200_ctx *c, int m, const int *idx, double *buf) {
  return eam_fp_call(c, m, idx, buf, true);
}

int b200_eam_fp_unpack(b200_ctx *c, int m, const int *idx, const double *buf) {
  return eam_fp_call(c, m, idx, const_cast<double *>(buf), false);
}

int b200_eam_force(b200_ctx *c, int eflag, int vflag, double *eng, double virial[6],
                   double *eatom, double *vatom) {
  int rc = eam_split_check(c);
  if (rc) return rc;
  if (c->eam_split_eflag != eflag || c->eam_split_vflag != vflag)
    return set_err(c, B200_ERR_STATE,
                   "b200_eam_force needs a b200_eam_density call with the same flags before it");
  c->eam_split_eflag = c->eam_split_vflag = -1;
  const bool eg = (eflag & 1) != 0, ea = (eflag & 2) != 0;
  const bool vg = (vflag % 4) != 0, va = (vflag & 4) != 0;
  const bool ev = eg || ea || vg || va;
  const int n = c->n;
  char *st[1];
  const size_t sb[1] = {(va && vatom) ? 6 * (size_t)n * sizeof(double) : 0};
  rc = xfer_parts(c, 1, sb, st);
  if (rc) return rc;
  double *dv = reinterpret_cast<double *>(st[0]);
  CK(md_eam_compute(c, ev, ea || va, ea ? c->eam_eatom : nullptr, dv, nullptr, EAM_FORCE));
  double h[8];
  if (ev) CK(cudaMemcpyAsync(h, c->ev, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (ea && eatom)
    CK(cudaMemcpyAsync(eatom, c->eam_eatom, (size_t)n * sizeof(double), cudaMemcpyDefault,
                       c->stream));
  if (dv) CK(cudaMemcpyAsync(vatom, dv, 6 * (size_t)n * sizeof(double), cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (ev) {
    if (eg && eng) *eng = h[0];
    if (vg && virial)
      for (int k = 0; k < 6; k++) virial[k] = h[1 + k];
  }
  return B200_OK;
}

int b200_nve_initial(b200_ctx *c, double dtv, double dtf) {
  if (!c) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  CK(md_nve_initial(c, dtv, dtf));
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

int b200_nve_final(b200_ctx *c, double dtf) {
  if (!c) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  CK(md_nve_final(c, dtf, false));
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

int b200_setup(b200_ctx *c, double *row) {
  if (!c) return B200_ERR_ARG;
  int rc = prepare(c);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->status, 0, ST_COUNT * sizeof(int), c->stream));
  rc = rebuild_sync(c);
  if (rc) return rc;
  c->sorted_once = true;
  // Verlet::setup resets the build counter after the setup build
  CK(cudaMemsetAsync(c->status + ST_NCALLS, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->status + ST_AGO, 0, sizeof(int), c->stream));
  if (c->tpa == 0 || !c->tuned) {
    if (c->tpa == 0) {
      rc = autotune(c);
      if (rc) return rc;
      // the step-form search leaves the state as it found it, so the first
      // run can repeat it between two of its steps
      c->retune_pending = step_form(c);
      c->retune_step = -1;
    }
    c->tuned = true;
  }
  if (c->nrep && !c->rep_tuned) {
    // forces first: the tuning steps run the half-steps on them
    rc = pair_compute_dev(c, false, false, nullptr, nullptr);
    if (!rc) rc = tune_replica_step(c);
    if (rc) return rc;
  }
  rc = pair_compute_dev(c, true, false, nullptr, nullptr);
  if (rc) return rc;
  CK(md_ke(c));
  double h[8];
  rc = small_read(c, h, c->ev, sizeof(h));
  if (rc) return rc;
  if (row) {
    row[0] = 0.0;
    row[1] = h[7];
    row[2] = h[0];
    for (int k = 0; k < 6; k++) row[3 + k] = h[1 + k];
  }
  return B200_OK;
}

int b200_run(b200_ctx *c, int nsteps, double dt, double ftm2v, int thermo_every, double *rows,
             int maxrows, int *nrows) {
  if (!c || nsteps < 0) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "b200_setup not called");
  if (c->ghosts_on)
    return set_err(c, B200_ERR_STATE,
                   "b200_run with ghost atoms: a decomposed box steps through the per-call entry "
                   "points and the halo exchange");
  CK(cudaSetDevice(c->device));
  const double dtv = dt, dtf = 0.5 * dt * ftm2v;  // FixNVE::init (src/fix_nve.cpp:52-59)
  // thermo rows: room for every output step of this run
  int nout = 1 + (thermo_every > 0 ? nsteps / thermo_every : 0);
  if (nout > c->rows_cap) {
    CK(dalloc(&c->rows, (size_t)9 * nout));
    c->rows_cap = nout;
    invalidate_graphs(c);
  }
  if (c->graph_valid && (c->graph_dt != dtv || c->graph_ftm2v != ftm2v || c->graph_tpa != c->tpa ||
                         c->graph_timing != c->timing))
    invalidate_graphs(c);
  const int chunk = 256;  // steps per timing read-back
  if (c->timing) {
    int rc = ensure_events(c, (size_t)(MD_NPHASE + 1) * chunk);
    if (rc) return rc;
  }
  // timing mode 2: two events around each piece, at most four pieces a step
  std::vector<signed char> piece_kind;
  if (c->timing_pieces) {
    int rc = ensure_events(c, (size_t)8 * chunk);
    if (rc) return rc;
    piece_kind.assign((size_t)4 * chunk, -1);
  }
  {
    int rc = ensure_graphs(c, dtv, dtf, ftm2v);
    if (rc) return rc;
  }
  CK(cudaMemsetAsync(c->status + ST_ROW, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->status + ST_OVERFLOW, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->status + ST_MAXNEIGH, 0, sizeof(int), c->stream));
  // host view of the current step for the output schedule
  int rc2 = read_status(c);
  if (rc2) return rc2;
  long long step0 = ((long long)(unsigned int)c->status_host[ST_STEP_HI] << 32) |
                    (long long)(unsigned int)c->status_host[ST_STEP_LO];
  const long long last = step0 + nsteps;
  long long s = step0 + 1;
  int replays = 0;
  bool force_build = false;
  // the one repeat of the launch-shape search, retune_steps steps into the
  // first run after the setup-time search, at a chunk boundary (whole
  // steps, forces stored)
  constexpr int retune_steps = 50;
  if (c->retune_pending && c->retune_step < 0) c->retune_step = step0 + retune_steps + 1;
  while (s <= last) {
    if (c->retune_pending && s >= c->retune_step) {
      int rc = autotune_step(c);
      if (rc) return rc;
      c->retune_pending = false;
      invalidate_graphs(c);
      rc = ensure_graphs(c, dtv, dtf, ftm2v);
      if (rc) return rc;
    }
    long long s_end = (last - s + 1) > chunk ? s + chunk - 1 : last;
    if (c->retune_pending && c->retune_step > s && c->retune_step - 1 < s_end)
      s_end = c->retune_step - 1;
    // A list that outgrows its capacity during a chunk is recovered by
    // replaying the chunk from this snapshot with a larger list, starting
    // with a forced rebuild (the reference instead stops with "Neighbor list
    // overflow, boost neigh_modify one", src/neigh_half_bin.cpp:414-415).
    int rc = snapshot(c, true);
    if (rc) return rc;
    const int ago0 = c->status_host[ST_AGO];
    auto is_out = [&](long long t) {
      return (t == last) || (thermo_every > 0 && t % thermo_every == 0);
    };
    // host mirror of Neighbor::ago (src/neighbor.cpp:1301-1309)
    int ago = c->status_host[ST_AGO];
    // Within a chunk (timers off) the final half-step of step t and the
    // initial half-step and decision of step t+1 run as one piece; a chunk
    // starts with its own initial half-step, so snapshots and replays see
    // whole steps.
    bool pre_done = false;
    if (c->timing_pieces) std::fill(piece_kind.begin(), piece_kind.end(), (signed char)-1);
    for (long long t = s; t <= s_end; t++) {
      cudaEvent_t *ev = c->timing ? &c->ev_pool[(size_t)(t - s) * (MD_NPHASE + 1)] : nullptr;
      // piece k of step t; timing mode 2 brackets it with two stream events
      auto piece = [&](int k, int kind, cudaEvent_t *pev) -> int {
        if (!c->timing_pieces) return run_piece(c, kind, dtv, dtf, pev);
        const size_t slot = (size_t)(t - s) * 4 + k;
        CK(cudaEventRecord(c->ev_pool[2 * slot], c->stream));
        const int r = run_piece(c, kind, dtv, dtf, nullptr);
        if (r) return r;
        CK(cudaEventRecord(c->ev_pool[2 * slot + 1], c->stream));
        piece_kind[slot] = (signed char)kind;
        return B200_OK;
      };
      if (!pre_done) rc = piece(0, PIECE_PRE, ev);
      if (rc) return rc;
      ago++;
      bool rebuild = false;
      if (force_build) {
        rebuild = true;  // replay after an overflow: the device decides the same
        force_build = false;
      } else if (ago >= c->delay && ago % c->every == 0) {
        if (!c->check) {
          rebuild = true;
        } else {
          // distance criterion: the decision the device just made (it
          // posts to the mailbox exactly on these steps)
          c->decisions++;
          rc = wait_decision(c, &rebuild);
          if (rc) return rc;
        }
      }
      if (rebuild) {
        rc = piece(1, PIECE_REBUILD, nullptr);
        if (rc) return rc;
        ago = 0;
      }
      const bool fuse = !c->timing && t < s_end;
      const int post = fuse ? (is_out(t) ? PIECE_FUSED_OUT : PIECE_FUSED)
                            : (is_out(t) ? PIECE_POST_OUT : PIECE_POST);
      rc = piece(2, post, ev ? ev + 2 : nullptr);
      if (rc) return rc;
      pre_done = fuse;
    }
    rc = read_status(c);
    if (rc) return rc;
    if (c->status_host[ST_LOST]) return status_errors(c);
    if (md_stage_feedback(c, c->status_host[ST_MAXSTAGE])) {
      // a builder tile staged more atoms than its shared memory held (it
      // took the slower global-memory path): larger staging from now on
      invalidate_graphs(c);
      rc = ensure_graphs(c, dtv, dtf, ftm2v);
      if (rc) return rc;
    }
    if (c->status_host[ST_OVERFLOW]) {
      if (c->one_user > 0 || ++replays > 4) return status_errors(c);
      const int need = c->status_host[ST_MAXNEIGH];
      int cap = (int)(need * 1.25) + 32;
      if (cap < c->capacity * 3 / 2) cap = c->capacity * 3 / 2;
      rc = grow_list(c, (cap + 7) & ~7, false);
      if (!rc) rc = snapshot(c, false);
      if (!rc) rc = ensure_graphs(c, dtv, dtf, ftm2v);
      if (rc) return rc;
      int one = 1;
      CK(cudaMemcpyAsync(c->status + ST_FORCE_BUILD, &one, sizeof(int), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaStreamSynchronize(c->stream));
      c->status_host[ST_AGO] = ago0;
      force_build = true;
      c->overflow_replays++;
      continue;
    }
    if (c->one_user <= 0 && c->status_host[ST_MAXNEIGH] * 20 > c->capacity * 17) {
      // within 15% of the capacity: widen the list for the next builds,
      // keeping the current entries (same stride, longer slab)
      int cap = ((int)(c->status_host[ST_MAXNEIGH] * 1.5) + 32 + 7) & ~7;
      rc = grow_list(c, cap, true);
      if (!rc) rc = ensure_graphs(c, dtv, dtf, ftm2v);
      if (rc) return rc;
    }
    if (c->timing_pieces) {
      // mode 2: phase 0 the initial half-step pieces (chunk starts), 1 the
      // rebuilds, 2 the force pieces with their half-steps (the one-launch
      // step for lj/cut)
      for (long long t = s; t <= s_end; t++) {
        float step = 0.f;
        for (int k = 0; k < 4; k++) {
          const size_t slot = (size_t)(t - s) * 4 + k;
          const int kind = piece_kind[slot];
          if (kind < 0) continue;
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, c->ev_pool[2 * slot], c->ev_pool[2 * slot + 1]));
          c->phase_ms[kind == PIECE_PRE ? 0 : (kind == PIECE_REBUILD ? 1 : 2)] += ms;
          step += ms;
        }
        c->step_ms.push_back(step);
      }
      c->phase_steps += s_end - s + 1;
    }
    if (c->timing) {
      for (long long t = s; t <= s_end; t++) {
        const size_t base = (size_t)(t - s) * (MD_NPHASE + 1);
        for (int k = 0; k < MD_NPHASE; k++) {
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, c->ev_pool[base + k], c->ev_pool[base + k + 1]));
          c->phase_ms[k] += ms;
        }
        float step = 0.f;
        CK(cudaEventElapsedTime(&step, c->ev_pool[base], c->ev_pool[base + MD_NPHASE]));
        c->step_ms.push_back(step);
      }
      c->phase_steps += s_end - s + 1;
    }
    s = s_end + 1;
  }
  int rc = read_status(c);
  if (rc) return rc;
  int nr = c->status_host[ST_ROW];
  if (nrows) *nrows = nr;
  if (rows && maxrows > 0 && nr > 0) {
    int cpy = nr < maxrows ? nr : maxrows;
    if (cpy > c->rows_cap) cpy = c->rows_cap;
    CK(cudaMemcpy(rows, c->rows, (size_t)9 * cpy * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return status_errors(c);
}

int b200_neigh_half(b200_ctx *c, int *numneigh, int *jowner, int *jimage, long long cap,
                    long long *total) {
  if (!c) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  const int n = c->n;
  int *dn = nullptr, *dj = nullptr, *di = nullptr;
  CK(cudaMalloc((void **)&dn, (size_t)n * sizeof(int)));
  if (cap > 0 && jowner && jimage) {
    CK(cudaMalloc((void **)&dj, (size_t)cap * sizeof(int)));
    CK(cudaMalloc((void **)&di, (size_t)cap * sizeof(int)));
  }
  long long tot = 0;
  cudaError_t e = md_half_list(c, dn, dj, di, dj ? cap : 0, &tot);
  if (e == cudaSuccess && numneigh)
    e = cudaMemcpy(numneigh, dn, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost);
  long long m = tot < cap ? tot : cap;
  if (e == cudaSuccess && dj && m > 0) {
    e = cudaMemcpy(jowner, dj, (size_t)m * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(jimage, di, (size_t)m * sizeof(int), cudaMemcpyDeviceToHost);
  }
  cudaFree(dn);
  if (dj) cudaFree(dj);
  if (di) cudaFree(di);
  if (e != cudaSuccess) return set_err(c, B200_ERR_CUDA, "half list: %s", cudaGetErrorString(e));
  if (total) *total = tot;
  return B200_OK;
}

int b200_neigh_stats(b200_ctx *c, long long *full_total, int *ncalls, int *ndanger, int *maxneigh,
                     int *capacity) {
  if (!c) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  unsigned long long h = 0;
  char *st[1];
  const size_t sb[1] = {sizeof(unsigned long long)};
  int rc = xfer_parts(c, 1, sb, st);
  if (rc) return rc;
  unsigned long long *d = reinterpret_cast<unsigned long long *>(st[0]);
  CK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream));
  k_full_total<<<md_blocks(c->n, 256), 256, 0, c->stream>>>(c->n, c->numneigh, d);
  c->launches++;
  CK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  if (full_total) *full_total = (long long)h;
  if (ncalls) *ncalls = c->status_host[ST_NCALLS];
  if (ndanger) *ndanger = c->status_host[ST_NDANGER];
  if (maxneigh) *maxneigh = c->status_host[ST_MAXNEIGH];
  if (capacity) *capacity = c->capacity;
  return B200_OK;
}

int b200_get_rho_fp(b200_ctx *c, double *rho, double *fp) {
  if (!c) return B200_ERR_ARG;
  if (c->pstyle != B200_PAIR_EAM) return set_err(c, B200_ERR_STATE, "pair style is not eam");
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  const int n = c->n;
  char *st[1];
  const size_t sb[1] = {(size_t)n * sizeof(double)};
  int rc = xfer_parts(c, 1, sb, st);
  if (rc) return rc;
  double *d = reinterpret_cast<double *>(st[0]);
  if (rho) {
    k_unsort_scalar<<<md_blocks(n, 256), 256, 0, c->stream>>>(n, c->orig, c->rho, d);
    CK(cudaMemcpyAsync(rho, d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  if (fp) {
    k_unsort_scalar<<<md_blocks(n, 256), 256, 0, c->stream>>>(n, c->orig, c->fp, d);
    CK(cudaMemcpyAsync(fp, d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  c->launches += 2;
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

int b200_set_launch(b200_ctx *c, int tpa, int block) {
  if (!c) return B200_ERR_ARG;
  if (!(tpa == 0 || tpa == 1 || tpa == 2 || tpa == 4 || tpa == 8 || tpa == 16 || tpa == 32))
    return set_err(c, B200_ERR_ARG, "threads per atom must be 0, 1, 2, 4, 8, 16 or 32");
  if (block != 0 && block != 128) return set_err(c, B200_ERR_ARG, "block size must be 128");
  c->tpa = tpa;
  c->tuned = tpa != 0;
  c->retune_pending = false;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_get_launch(const b200_ctx *c, int *tpa, int *block) {
  if (!c) return B200_ERR_ARG;
  if (tpa) *tpa = c->tpa;
  if (block) *block = c->block;
  return B200_OK;
}

long long b200_kernel_launches(const b200_ctx *c) { return c ? c->launches : 0; }

int b200_set_timing(b200_ctx *c, int on) {
  if (!c || on < 0 || on > 2) return B200_ERR_ARG;
  c->timing = on == 1;
  c->timing_pieces = on == 2;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_set_graphs(b200_ctx *c, int on) {
  if (!c) return B200_ERR_ARG;
  c->use_graphs = on != 0;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_get_timing(b200_ctx *c, double *phase_ms, long long *steps, int reset) {
  if (!c) return B200_ERR_ARG;
  if (phase_ms)
    for (int k = 0; k < MD_NPHASE; k++) phase_ms[k] = c->phase_ms[k];
  if (steps) *steps = c->phase_steps;
  if (reset) {
    for (int k = 0; k < MD_NPHASE; k++) c->phase_ms[k] = 0.0;
    c->phase_steps = 0;
  }
  return B200_OK;
}

void *b200_stream(const b200_ctx *c) { return c ? (void *)c->stream : nullptr; }

int b200_get_step_times(b200_ctx *c, double *ms, int cap, int *count, int reset) {
  if (!c) return B200_ERR_ARG;
  const int n = (int)c->step_ms.size();
  if (count) *count = n;
  if (ms)
    for (int k = 0; k < n && k < cap; k++) ms[k] = c->step_ms[k];
  if (reset) c->step_ms.clear();
  return B200_OK;
}

}  // extern "C"

// ---- force matching --------------------------------------------------------

namespace {
int adj_check(b200_ctx *c, const double *lj1, const double *lj2, const double *cutsq) {
  if (!c || !lj1 || !lj2 || !cutsq) return B200_ERR_ARG;
  if (c->pstyle != B200_PAIR_LJ_CUT) return set_err(c, B200_ERR_STATE, "force matching needs lj/cut");
  if (c->ntypes > MD_ADJ_MAXTYPES)
    return set_err(c, B200_ERR_ARG, "force matching supports at most %d types", MD_ADJ_MAXTYPES);
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  const int w = c->ntypes + 1;
  for (int a = 1; a <= c->ntypes; a++)
    for (int b = 1; b <= c->ntypes; b++) {
      const double cs = cutsq[a * w + b];
      if (!(cs >= 0.0) || cs > c->cutneighsq[a * w + b])
        return set_err(c, B200_ERR_ARG,
                       "cutoff of types %d,%d beyond the neighbor list (set_lj, then build)", a, b);
    }
  CK(cudaSetDevice(c->device));
  return B200_OK;
}
}  // namespace

int b200_adj_set_positions(b200_ctx *c, const double *x) {
  if (!c || !x) return B200_ERR_ARG;
  if (!c->have_atoms) return set_err(c, B200_ERR_STATE, "no atoms uploaded");
  CK(cudaSetDevice(c->device));
  CK(md_adj_positions(c, x));
  int rc = prepare(c);
  if (rc) return rc;
  rc = rebuild_sync(c);
  if (rc) return rc;
  c->sorted_once = true;
  return B200_OK;
}

int b200_adj_forces(b200_ctx *c, const double *lj1, const double *lj2, const double *cutsq,
                    double *f) {
  int rc = adj_check(c, lj1, lj2, cutsq);
  if (rc) return rc;
  if (!f) return set_err(c, B200_ERR_ARG, "null force array");
  CK(md_adj_forward(c, lj1, lj2, cutsq, f));
  CK(cudaStreamSynchronize(c->stream));
  return B200_OK;
}

int b200_adj_backward(b200_ctx *c, const double *lj1, const double *lj2, const double *cutsq,
                      const double *g, double *gx, double *glj1, double *glj2) {
  int rc = adj_check(c, lj1, lj2, cutsq);
  if (rc) return rc;
  if (!g || !gx) return set_err(c, B200_ERR_ARG, "null gradient array");
  if (c->adj_n < c->n) {
    CK(dalloc(&c->adj_gs, 3 * (size_t)c->stride));
    c->adj_n = c->stride;
  }
  if (!c->adj_gtab) CK(dalloc(&c->adj_gtab, 2 * MD_ADJ_MAXTYPES * MD_ADJ_MAXTYPES));
  CK(md_adj_backward(c, lj1, lj2, cutsq, g, gx, c->adj_gs, c->adj_gtab));
  double h[2 * MD_ADJ_MAXTYPES * MD_ADJ_MAXTYPES];
  CK(cudaMemcpyAsync(h, c->adj_gtab, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int w = c->ntypes + 1;
  for (int k = 0; k < w * w; k++) {
    if (glj1) glj1[k] = 0.0;
    if (glj2) glj2[k] = 0.0;
  }
  for (int a = 1; a <= c->ntypes; a++)
    for (int b = 1; b <= c->ntypes; b++) {
      const int p = (a - 1) * c->ntypes + (b - 1);
      if (glj1) glj1[a * w + b] = h[2 * p];
      if (glj2) glj2[a * w + b] = h[2 * p + 1];
    }
  return B200_OK;
}

// ---- replicas --------------------------------------------------------------

// ---- spatial decomposition: ghosts, distance check, halo ----------------------

int b200_set_ghosts(b200_ctx *c, const int *ghost) {
  if (!c) return B200_ERR_ARG;
  if (!c->have_atoms) return set_err(c, B200_ERR_STATE, "no atoms uploaded");
  if (c->nrep) return set_err(c, B200_ERR_STATE, "ghost atoms with replicas");
  CK(cudaSetDevice(c->device));
  if (!ghost) {
    c->ghosts_on = false;
    return B200_OK;
  }
  CK(cudaMemcpyAsync(c->ghost, ghost, (size_t)c->n * sizeof(int), cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->ghosts_on = true;
  return B200_OK;
}

int b200_neigh_check(b200_ctx *c, int *moved) {
  if (!c || !moved) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->status_host + ST_MOVED, c->status + ST_MOVED, sizeof(int),
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(c->status + ST_MOVED, 0, sizeof(int), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *moved = c->status_host[ST_MOVED] != 0;
  return B200_OK;
}

static int halo_call(b200_ctx *c, int m, const int *idx, const double *buf, bool pack) {
  if (!c || m < 0 || (m > 0 && (!idx || !buf))) return B200_ERR_ARG;
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  if (m == 0) return B200_OK;
  CK(cudaMemsetAsync(c->status + ST_HALO_BAD, 0, sizeof(int), c->stream));
  if (pack)
    CK(md_halo_pack(c, m, idx, const_cast<double *>(buf)));
  else
    CK(md_halo_unpack(c, m, idx, buf));
  int rc = read_status(c);
  if (rc) return rc;
  if (c->status_host[ST_HALO_BAD] == 2)
    return set_err(c, B200_ERR_ARG, "halo unpack: an index names an owned atom, not a ghost");
  if (c->status_host[ST_HALO_BAD])
    return set_err(c, B200_ERR_ARG, "halo %s: an atom index is outside [0, %d)",
                   pack ? "pack" : "unpack", c->n);
  return B200_OK;
}

int b200_halo_pack(b200_ctx *c, int m, const int *idx, double *buf) {
  return halo_call(c, m, idx, buf, true);
}

int b200_halo_unpack(b200_ctx *c, int m, const int *idx, const double *buf) {
  return halo_call(c, m, idx, buf, false);
}

int b200_set_replicas(b200_ctx *c, int nrep, const int *natoms, const double *lo,
                      const double *hi) {
  if (!c || nrep < 1 || !natoms || !lo || !hi) return B200_ERR_ARG;
  long long total = 0;
  for (int r = 0; r < nrep; r++) {
    if (natoms[r] < 1) return set_err(c, B200_ERR_ARG, "replica %d has no atoms", r);
    for (int d = 0; d < 3; d++)
      if (!(hi[3 * r + d] > lo[3 * r + d]))
        return set_err(c, B200_ERR_ARG, "replica %d: box hi <= lo in dim %d", r, d);
    total += natoms[r];
  }
  if (total > MD_MAX_ATOMS) return set_err(c, B200_ERR_ARG, "too many atoms (%lld)", total);
  c->nrep = nrep;
  c->rep_natoms.assign(natoms, natoms + nrep);
  c->rep_atom_start.assign(nrep + 1, 0);
  for (int r = 0; r < nrep; r++) c->rep_atom_start[r + 1] = c->rep_atom_start[r] + natoms[r];
  c->rep_lo.assign(lo, lo + 3 * nrep);
  c->rep_hi.assign(hi, hi + 3 * nrep);
  c->rep_box.assign(nrep, BoxGeom{});
  for (int r = 0; r < nrep; r++)
    for (int d = 0; d < 3; d++) {
      c->rep_box[r].lo[d] = lo[3 * r + d];
      c->rep_box[r].hi[d] = hi[3 * r + d];
      c->rep_box[r].prd[d] = hi[3 * r + d] - lo[3 * r + d];  // Domain::set_global_box
    }
  c->box = c->rep_box[0];
  c->box_set = true;
  c->sorted_once = false;
  c->rep_tuned = false;  // a new batch: its step form is chosen again
  invalidate_graphs(c);
  return B200_OK;
}

int b200_replica_count(const b200_ctx *c) { return c ? c->nrep : 0; }

int b200_set_replica_step(b200_ctx *c, int mode, int cluster, int block, int tpa) {
  if (!c || mode < 0 || mode > 2 || !(cluster == 0 || cluster == 1 || cluster == 2 || cluster == 4) ||
      !(block == 0 || block == 256 || block == 512) || !(tpa == 0 || tpa == 1 || tpa == 2 || tpa == 4))
    return set_err(c, B200_ERR_ARG, "Illegal replica step form");
  c->rep_mode = mode;
  c->rep_fix_cs = cluster;
  c->rep_fix_block = block;
  c->rep_fix_tpa = tpa;
  c->rep_onelaunch = false;  // decided again by the next b200_setup
  c->rep_tuned = false;
  invalidate_graphs(c);
  return B200_OK;
}

int b200_get_replica_step(const b200_ctx *c, int *onelaunch, int *cluster, int *block, int *tpa,
                          double *ms) {
  if (!c) return B200_ERR_ARG;
  if (onelaunch) *onelaunch = c->rep_onelaunch ? 1 : 0;
  if (cluster) *cluster = c->rep_cs;
  if (block) *block = c->rep_block;
  if (tpa) *tpa = c->rep_tpa;
  if (ms) {
    ms[0] = c->rep_tune_ms[0];
    ms[1] = c->rep_tune_ms[1];
  }
  return B200_OK;
}

int b200_replica_thermo(b200_ctx *c, double *rows) {
  if (!c || !rows) return B200_ERR_ARG;
  if (!c->nrep) return set_err(c, B200_ERR_STATE, "no replicas set");
  if (!c->sorted_once) return set_err(c, B200_ERR_STATE, "neighbor list not built");
  CK(cudaSetDevice(c->device));
  const int n = c->n, R = c->nrep;
  char *st[4];
  const size_t sb[4] = {(size_t)n * sizeof(double), 6 * (size_t)n * sizeof(double),
                        9 * (size_t)R * sizeof(double), ((size_t)R + 1) * sizeof(int)};
  int rc = xfer_parts(c, 4, sb, st);
  if (rc) return rc;
  double *eatom = reinterpret_cast<double *>(st[0]), *vatom = reinterpret_cast<double *>(st[1]);
  double *drows = reinterpret_cast<double *>(st[2]);
  int *d_start = reinterpret_cast<int *>(st[3]);
  CK(cudaMemcpyAsync(d_start, c->rep_atom_start.data(), ((size_t)R + 1) * sizeof(int),
                     cudaMemcpyHostToDevice, c->stream));
  rc = pair_compute_dev(c, true, true, eatom, vatom);
  if (!rc) {
    cudaError_t e = md_rep_rows(c, d_start, eatom, vatom, drows);
    if (e != cudaSuccess) rc = set_err(c, B200_ERR_CUDA, "replica rows: %s", cudaGetErrorString(e));
  }
  if (!rc)
    CK(cudaMemcpyAsync(rows, drows, 9 * (size_t)R * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return rc;
}
