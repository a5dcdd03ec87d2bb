// neigh.cu -- device rebuild of the cell-sorted atom order and the full
// neighbor list, plus export of the reference's half list.
//
// Rebuild (every `every` steps, or when an atom moved more than half the
// skin) replaces Domain::pbc (src/domain.cpp:478-560), Atom::sort
// (src/atom.cpp:1575-1700), CommBrick::borders (src/comm_brick.cpp:696-864)
// and Neighbor::build -> half_bin_newton (src/neigh_half_bin.cpp:285-419):
//   1 k_wrap_bin    wrap into the box (image flags), count atoms per cell
//   2 k_scan_*      exclusive scan of the counts -> cell_start
//   3 k_scatter     counting-sort scatter of atom indices; zeroes the counts
//   4 k_sort_cells  order each cell by caller index (deterministic order)
//   5 k_gather      permute x, v, ids; fixed-point copy (mixed); xhold
//   6 k_copyback    permuted arrays back into the primary buffers, the
//                   caller-index -> slot map; ago = 0
//   7 k_neigh_tiles full list over the 27 neighbor cells (cell >= rc+skin),
//                   neighbor-cell tiles staged in shared memory
// The pair test is the reference's, bit for bit: the periodic image is
// formed as x_j + s*L in FP64 and rsq = dx*dx + dy*dy + dz*dz is rounded
// after every operation, then compared with `<=` to (rc+skin)^2
// (src/neigh_half_bin.cpp:355-360, src/atom_vec_atomic.cpp:297-299).
#include <cstdio>

#include "md_state.h"

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ bool rebuild_on(const int *flag) { return flag == nullptr || *flag != 0; }

template <bool BATCH>
__global__ void k_wrap_bin(int n, BoxGeom box1, Reps reps, double4 *__restrict__ x4,
                           int *__restrict__ image, int *__restrict__ cell_count,
                           int *__restrict__ slot, int *__restrict__ cell_tmp,
                           int *__restrict__ status, const int *flag) {
  if (!rebuild_on(flag)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int rep = BATCH ? reps.rep_of_atom[i] : 0;
  const BoxGeom &box = BATCH ? reps.box[rep] : box1;
  double4 p = x4[i];
  double xs[3] = {p.x, p.y, p.z};
  int img = image[i];
  int im[3] = {(img & MD_IMGMASK) - MD_IMGMAX, ((img >> 10) & MD_IMGMASK) - MD_IMGMAX,
               ((img >> 20) & MD_IMGMASK) - MD_IMGMAX};
  int cc[3];
  bool bad = false;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double x = xs[d];
    if (!isfinite(x)) {
      bad = true;
      x = box.lo[d];
    }
    // Domain::pbc: x < lo -> x += prd; x >= hi -> x -= prd, x = max(x, lo)
    if (x < box.lo[d]) {
      x = __dadd_rn(x, box.prd[d]);
      im[d]--;
    }
    if (x >= box.hi[d]) {
      x = __dsub_rn(x, box.prd[d]);
      x = fmax(x, box.lo[d]);
      im[d]++;
    }
    if (x < box.lo[d] || x >= box.hi[d]) bad = true;
    xs[d] = x;
    int c = (int)((x - box.lo[d]) * box.cinv[d]);
    c = c < 0 ? 0 : (c >= box.ncell[d] ? box.ncell[d] - 1 : c);
    cc[d] = c;
  }
  if (bad) atomicExch(&status[ST_LOST], 1);
  x4[i] = make_double4(xs[0], xs[1], xs[2], p.w);
  image[i] = md_img_pack(im[0], im[1], im[2]);
  int c = cc[0] + box.ncell[0] * (cc[1] + box.ncell[1] * cc[2]);
  if (BATCH) c += reps.cell_base[rep];
  slot[i] = atomicAdd(&cell_count[c], 1);
  cell_tmp[i] = c;
}

// block-wide exclusive scan of kScanTile ints; block sums to `sums`
__global__ void k_scan_tiles(int m, const int *__restrict__ in, int *__restrict__ out,
                             int *__restrict__ sums, const int *flag) {
  if (!rebuild_on(flag)) return;
  __shared__ int warp_tot[kScanThreads / 32];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int run = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    int idx = base + k;
    int a = idx < m ? in[idx] : 0;
    v[k] = run;
    run += a;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int t = warp_tot[lane];
    int s = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += u;
    }
    warp_tot[lane] = s - t;  // exclusive prefix of warp totals
    if (lane == 31 && sums) sums[blockIdx.x] = s;
  }
  __syncthreads();
  int excl = incl - run + warp_tot[warp];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    int idx = base + k;
    if (idx < m) out[idx] = v[k] + excl;
  }
}

__global__ void k_scan_add(int m, int *__restrict__ out, const int *__restrict__ sums,
                           const int *flag) {
  if (!rebuild_on(flag)) return;
  int b = blockIdx.x;
  if (b == 0) return;
  int add = sums[b];
  int base = b * kScanTile;
  for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
    int idx = base + k;
    if (idx < m) out[idx] += add;
  }
}

// Scatter each atom to its slot in the cell-sorted order.  The scan has
// consumed the m cell counts by now, so this kernel also zeroes them for the
// next build (the counts start at zero when they are allocated).
__global__ void k_scatter(int n, const int *__restrict__ cell_tmp, const int *__restrict__ slot,
                          const int *__restrict__ cell_start, int *__restrict__ perm, int m,
                          int *__restrict__ cell_count, const int *flag) {
  if (!rebuild_on(flag)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = i; k < m; k += gridDim.x * blockDim.x) cell_count[k] = 0;
  if (i >= n) return;
  perm[cell_start[cell_tmp[i]] + slot[i]] = i;
}

// One warp per cell: rank the cell's atoms by caller index so that the
// sorted order (and with it every summation order) is reproducible.
constexpr int kSortWarps = 8;
constexpr int kSortSmall = 64;

__global__ void k_sort_cells(int ncells, const int *__restrict__ cell_start, int *__restrict__ perm,
                             int *__restrict__ tmp, const int *__restrict__ orig, const int *flag) {
  if (!rebuild_on(flag)) return;
  __shared__ int skey[kSortWarps][kSortSmall];
  __shared__ int sval[kSortWarps][kSortSmall];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int c = blockIdx.x * kSortWarps + w;
  if (c >= ncells) return;
  int s = cell_start[c], e = cell_start[c + 1], cnt = e - s;
  if (cnt <= 1) return;
  if (cnt <= kSortSmall) {
    for (int k = lane; k < cnt; k += 32) {
      int val = perm[s + k];
      sval[w][k] = val;
      skey[w][k] = orig[val];
    }
    __syncwarp();
    for (int k = lane; k < cnt; k += 32) {
      int key = skey[w][k], r = 0;
      for (int m = 0; m < cnt; m++) r += skey[w][m] < key;
      perm[s + r] = sval[w][k];
    }
  } else {
    for (int k = lane; k < cnt; k += 32) tmp[s + k] = perm[s + k];
    __threadfence_block();
    __syncwarp();
    for (int k = lane; k < cnt; k += 32) {
      int val = tmp[s + k], key = orig[val], r = 0;
      for (int m = 0; m < cnt; m++) r += orig[tmp[s + m]] < key;
      perm[s + r] = val;
    }
  }
}

template <bool BATCH>
__global__ void k_gather(int n, int stride, BoxGeom box1, Reps reps, const int *__restrict__ perm,
                         const double4 *__restrict__ x4, double4 *__restrict__ x4b,
                         const double *__restrict__ v, double *__restrict__ vb,
                         const int *__restrict__ orig, int *__restrict__ origb,
                         const int *__restrict__ image, int *__restrict__ imageb,
                         const int *__restrict__ cell_tmp, int *__restrict__ cell,
                         int4 *__restrict__ xq, double4 *__restrict__ xhold, const int *flag) {
  if (!rebuild_on(flag)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int old = perm[k];
  double4 p = x4[old];
  x4b[k] = p;
  vb[k] = v[old];
  vb[stride + k] = v[stride + old];
  vb[2 * stride + k] = v[2 * stride + old];
  origb[k] = orig[old];
  imageb[k] = image[old];
  int c = cell_tmp[old];
  const int rep = BATCH ? reps.rep_of_atom[k] : 0;
  const BoxGeom &box = BATCH ? reps.box[rep] : box1;
  if (BATCH) c -= reps.cell_base[rep];
  int cx = c % box.ncell[0];
  int cy = (c / box.ncell[0]) % box.ncell[1];
  int cz = c / (box.ncell[0] * box.ncell[1]);
  cell[k] = md_cell_pack(cx, cy, cz);
  if (xhold) xhold[k] = p;
  if (xq) xq[k] = md_xq(p, box);
}

__global__ void k_copyback(int n, int stride, const double4 *__restrict__ x4b,
                           double4 *__restrict__ x4, const double *__restrict__ vb,
                           double *__restrict__ v, const int *__restrict__ origb,
                           int *__restrict__ orig, const int *__restrict__ imageb,
                           int *__restrict__ image, int *__restrict__ where,
                           int *__restrict__ status, const int *flag) {
  if (!rebuild_on(flag)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0) {
    // Neighbor::build bookkeeping: ago = 0, ncalls++ (src/neighbor.cpp:1384-1386)
    status[ST_AGO] = 0;
    status[ST_NCALLS] += 1;
  }
  if (k >= n) return;
  x4[k] = x4b[k];
  v[k] = vb[k];
  v[stride + k] = vb[stride + k];
  v[2 * stride + k] = vb[2 * stride + k];
  const int o = origb[k];
  orig[k] = o;
  where[o] = k;  // caller index -> sorted slot, for the halo pack / unpack
  image[k] = imageb[k];
}

// Full neighbor list with shared-memory staging of neighbor-cell tiles.
// A CTA owns kTileCells consecutive cells along x; the 3 x 3 x (kTileCells+2)
// block of cells around them is staged in shared memory as 9 contiguous
// ranges of the cell-sorted atom arrays (positions as FP32 offsets from the
// CTA's reference point, with the periodic image already applied).  Each
// thread takes one atom of the owned cells and scans its 27 neighbor cells
// from shared memory.  The FP32 distance decides every pair whose rsq lies
// outside a relative band of 1e-5 around (rc+skin)^2; pairs inside the band
// are decided by the reference's FP64 arithmetic on the global FP64
// positions, so the list is bit-identical to the FP64 criterion.
constexpr int kTileCells = MD_TILE_CELLS;
// staged atoms per tile at most: 8192 x 16 B = 128 KB of shared memory, with
// the opt-in above the default 48 KB (set on the first build)
constexpr int kStageCapMax = 8192;
constexpr int kStageCells = 3 * 3 * (kTileCells + 2);
constexpr int kNeighThreads = 32 * kTileCells;  // one warp per owned cell

// The last four list entries of a thread rotate through an int4 register
// buffer; every fourth append stores the slab with one 16-byte write.
__device__ __forceinline__ void append_entry(int *__restrict__ nlist, int stride, int i,
                                             int &count, int capacity, int e, int4 &buf) {
  buf.x = buf.y;
  buf.y = buf.z;
  buf.z = buf.w;
  buf.w = e;
  if ((count & 3) == 3 && count < capacity)
    reinterpret_cast<int4 *>(nlist)[(size_t)(count >> 2) * stride + i] = buf;
  count++;
}

// store the last, partly filled slab (its r entries sit at the end of buf;
// the rest of the slab is filled with the atom's pad entry)
__device__ __forceinline__ void flush_entries(int *__restrict__ nlist, int stride, int i,
                                              int count, int capacity, const int4 &buf) {
  const int r = count & 3;
  if (r == 0 || count - 1 >= capacity) return;
  const int pad = md_pad_entry(i);
  int4 o = make_int4(pad, pad, pad, pad);
  if (r == 1) o.x = buf.w;
  else if (r == 2) { o.x = buf.z; o.y = buf.w; }
  else { o.x = buf.y; o.y = buf.z; o.z = buf.w; }
  reinterpret_cast<int4 *>(nlist)[(size_t)(count >> 2) * stride + i] = o;
}

// exact reference criterion for one candidate (FP64, no contraction)
__device__ __forceinline__ bool exact_pair(const double4 &xi, const double4 &xj, double shx,
                                           double shy, double shz, double cutsq) {
  const double delx = __dsub_rn(xi.x, __dadd_rn(xj.x, shx));
  const double dely = __dsub_rn(xi.y, __dadd_rn(xj.y, shy));
  const double delz = __dsub_rn(xi.z, __dadd_rn(xj.z, shz));
  return dsq3(delx, dely, delz) <= cutsq;
}

// Shared memory of k_neigh_tiles: stage_cap + 32 float4 staged atoms (32
// spare slots: a chunk may read past a row).  The .w word of a staged atom
// packs its list entry and type: bits 6..31 the atom index, bits 3..5 the
// type minus one, bits 0..2 the staged column sx (0 .. kTileCells+1).
static size_t neigh_smem(int stage_cap) { return (size_t)(stage_cap + 32) * sizeof(float4); }

__device__ __forceinline__ int stage_word(int j, int type, int sx) {
  return (int)(((unsigned)j << 6) | ((unsigned)(type - 1) << 3) | (unsigned)sx);
}
__device__ __forceinline__ int stage_type(float w) { return ((__float_as_int(w) >> 3) & 7) + 1; }
// the list entry (j << 6 | sx) of a staged atom
__device__ __forceinline__ unsigned stage_entry(float w) {
  return (unsigned)__float_as_int(w) & ~0x38u;
}

template <bool SINGLE, bool BATCH>
__global__ void __launch_bounds__(kNeighThreads, 8) k_neigh_tiles(
    int n, int stride, int capacity, int stage_cap, BoxGeom box1, Reps reps, int ntp1,
    const double *__restrict__ cutneighsq_g, const double4 *__restrict__ x4,
    const int *__restrict__ cell_start_g, int *__restrict__ nlist, int *__restrict__ numneigh,
    int *__restrict__ status, const int *flag, int pass, int cap1) {
  if (!rebuild_on(flag)) return;
  // batched: this tile's replica, its box and its cells' slice of cell_start
  const int rep = BATCH ? reps.tile_rep[blockIdx.x] : 0;
  const int tile = BATCH ? blockIdx.x - reps.tile_base[rep] : blockIdx.x;
  const BoxGeom &box = BATCH ? reps.box[rep] : box1;
  const int *__restrict__ cell_start = BATCH ? cell_start_g + reps.cell_base[rep] : cell_start_g;
  extern __shared__ float4 s_stage[];
  float4 *sp = s_stage;
  __shared__ int s_start[kStageCells + 1];
  __shared__ int s_src[kStageCells];
  __shared__ double s_sh[kStageCells][3];
  __shared__ double cns[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  __shared__ float cns_lo[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  __shared__ float cns_hi[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  const int ncx = box.ncell[0], ncy = box.ncell[1], ncz = box.ncell[2];
  const int tiles_x = (ncx + kTileCells - 1) / kTileCells;
  const int bx = tile % tiles_x;
  const int cy = (tile / tiles_x) % ncy;
  const int cz = tile / (tiles_x * ncy);
  const int cx0 = bx * kTileCells;
  const int ow = min(kTileCells, ncx - cx0);  // owned cells in this tile
  for (int k = threadIdx.x; k < ntp1 * ntp1; k += blockDim.x) {
    const double c = cutneighsq_g[k];
    cns[k] = c;
    cns_lo[k] = (float)(c * (1.0 - 1.0e-5));
    cns_hi[k] = (float)(c * (1.0 + 1.0e-5));
  }
  // staged cells: id = sx + (kTileCells+2)*(sy + 3*sz) is global cell
  // (cx0-1+sx, cy-1+sy, cz-1+sz), wrapped, with the shift of its image
  if (threadIdx.x < kStageCells) {
    const int id = threadIdx.x;
    const int sx = id % (kTileCells + 2), sy = (id / (kTileCells + 2)) % 3,
              sz = id / (3 * (kTileCells + 2));
    int g = 0, ix = 0, iy = 0, iz = 0, cnt = 0;
    if (sx <= ow + 1) {  // columns past the box edge are not neighbours of any owned cell
      int gx = cx0 - 1 + sx, gy = cy - 1 + sy, gz = cz - 1 + sz;
      if (gx < 0) { gx += ncx; ix = -1; } else if (gx >= ncx) { gx -= ncx; ix = 1; }
      if (gy < 0) { gy += ncy; iy = -1; } else if (gy >= ncy) { gy -= ncy; iy = 1; }
      if (gz < 0) { gz += ncz; iz = -1; } else if (gz >= ncz) { gz -= ncz; iz = 1; }
      g = gx + ncx * (gy + ncy * gz);
      cnt = cell_start[g + 1] - cell_start[g];
    }
    s_src[id] = g;
    s_sh[id][0] = ix * box.prd[0];
    s_sh[id][1] = iy * box.prd[1];
    s_sh[id][2] = iz * box.prd[2];
    s_start[id + 1] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s_start[0] = 0;
    for (int id = 0; id < kStageCells; id++) s_start[id + 1] += s_start[id];
  }
  __syncthreads();
  // pass 0: every tile (staged, or the global-memory path when it does not
  // fit); pass 1: the tiles that fit stage_cap; pass 2: only the tiles that
  // pass 1 left (more than cap1 atoms), with a larger stage_cap
  const int nstage = s_start[kStageCells];
  if ((pass == 1 && nstage > stage_cap) || (pass == 2 && nstage <= cap1)) return;
  const bool staged = nstage <= stage_cap;
  if (threadIdx.x == 0) atomicMax(&status[ST_MAXSTAGE], nstage);
  // FP32 reference point: centre of cell (cx0, cy, cz)
  const double rx = box.lo[0] + (cx0 + 0.5) * box.cs[0];
  const double ry = box.lo[1] + (cy + 0.5) * box.cs[1];
  const double rz = box.lo[2] + (cz + 0.5) * box.cs[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (staged) {
    for (int id = warp; id < kStageCells; id += kNeighThreads / 32) {
      const int g0 = cell_start[s_src[id]];
      const int cnt = s_start[id + 1] - s_start[id];
      const double shx = s_sh[id][0], shy = s_sh[id][1], shz = s_sh[id][2];
      for (int t = lane; t < cnt; t += 32) {
        const double4 p = x4[g0 + t];
        const int o = s_start[id] + t;
        sp[o] = make_float4((float)(__dadd_rn(p.x, shx) - rx), (float)(__dadd_rn(p.y, shy) - ry),
                            (float)(__dadd_rn(p.z, shz) - rz),
                            __int_as_float(stage_word(g0 + t, (int)p.w, id % (kTileCells + 2))));
      }
    }
  }
  // the spare slots after the last staged row: far away, type 1
  if (staged && threadIdx.x < 32)
    sp[s_start[kStageCells] + threadIdx.x] =
        make_float4(1.0e30f, 1.0e30f, 1.0e30f, __int_as_float(stage_word(0, 1, 0)));
  __syncthreads();
  // Warp w owns cell (cx0 + w, cy, cz); each lane takes one of its atoms.
  // The 27 neighbour cells are 9 contiguous staged ranges (3 cells along x
  // each), scanned 32 candidates at a time.  Test phase: each lane holds one
  // candidate and the warp steps through the owned atoms (broadcast shared
  // reads); one ballot per owned atom gives that atom's 32-bit acceptance
  // mask, which the atom's own lane keeps.  Append phase: each lane walks the
  // set bits of its mask in candidate order.
  if (warp >= ow) return;
  const int own_id = (warp + 1) + (kTileCells + 2) * (1 + 3 * 1);
  const int cown = cx0 + warp + ncx * (cy + ncy * cz);
  const int a0 = cell_start[cown], a1 = cell_start[cown + 1];
  const float lo1 = SINGLE ? cns_lo[ntp1 + 1] : 0.f, hi1 = SINGLE ? cns_hi[ntp1 + 1] : 0.f;
  const double cut1 = SINGLE ? cns[ntp1 + 1] : 0.0;
  if (staged) {
    const int o0 = s_start[own_id];
    for (int base = a0; base < a1; base += 32) {
      const int i = base + lane;
      const bool act = i < a1;
      // the FP64 position is read again only for a pair in the FP32 band
      const int ti = SINGLE ? 1 : (int)x4[act ? i : a0].w;
      const int my_m = act ? o0 + (i - a0) : -1;
      // the owned atoms of this batch, staged as sp[ob .. ob + na) with the
      // same FP32 offsets from the tile centre as every candidate
      const int ob = o0 + (base - a0), na = min(32, a1 - base);
      int count = 0;
      int4 buf = make_int4(0, 0, 0, 0);
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++) {
          const int idL = warp + (kTileCells + 2) * ((1 + dy) + 3 * (1 + dz));  // dx = -1
          const int r0 = s_start[idL], r1 = s_start[idL + 3];
          // entry code of a candidate in staged column sx: dx + 1 = sx - warp
          const unsigned rowadd = (unsigned)(((dy + 1) << 2) + ((dz + 1) << 4) - warp);
          for (int cb = r0; cb < r1; cb += 32) {
            const int nc = min(32, r1 - cb);
            // this lane's candidate (the spare slots past the last row are
            // far away, and candidates past the row end are masked below)
            const float4 pc = sp[cb + lane];
            const int tc = stage_type(pc.w);
            unsigned acc = 0u, band = 0u;
            for (int a = 0; a < na; a++) {
              const float4 q = sp[ob + a];
              const float ddx = q.x - pc.x, ddy = q.y - pc.y, ddz = q.z - pc.z;
              const float r2 = ddx * ddx + ddy * ddy + ddz * ddz;
              float lo = lo1, hi = hi1;
              if (!SINGLE) {
                const int tt = stage_type(q.w) * ntp1 + tc;
                lo = cns_lo[tt];
                hi = cns_hi[tt];
              }
              const bool in = r2 <= hi;
              const unsigned m = __ballot_sync(0xffffffffu, in);
              const unsigned b = __ballot_sync(0xffffffffu, in && r2 >= lo);
              if (lane == a) {
                acc = m;
                band = b;
              }
            }
            // candidates past the row end are not neighbours
            acc &= nc == 32 ? 0xffffffffu : ((1u << nc) - 1u);
            if (my_m >= cb && my_m < cb + nc) acc &= ~(1u << (my_m - cb));
            band &= acc;
            if (band == 0u) {
              while (acc) {
                const int t = __ffs(acc) - 1;
                acc &= acc - 1u;
                append_entry(nlist, stride, i, count, capacity,
                             (int)(stage_entry(sp[cb + t].w) + rowadd), buf);
              }
            } else {
              while (acc) {
                const int t = __ffs(acc) - 1;
                acc &= acc - 1u;
                const int m = cb + t;
                const unsigned bits = stage_entry(sp[m].w);
                // inside the FP32 uncertainty band: the reference's FP64 test
                if ((band >> t) & 1u) {
                  const int id = idL - warp + (int)(bits & 7u);
                  if (!exact_pair(x4[i], x4[md_entry_j(bits)], s_sh[id][0], s_sh[id][1], s_sh[id][2],
                                  SINGLE ? cut1 : cns[ti * ntp1 + stage_type(sp[m].w)]))
                    continue;
                }
                append_entry(nlist, stride, i, count, capacity, (int)(bits + rowadd), buf);
              }
            }
          }
        }
      if (act) {
        flush_entries(nlist, stride, i, count, capacity, buf);
        // the stored count never exceeds the capacity, so readers stay in
        // bounds; an overflow is reported through the status word
        numneigh[i] = count < capacity ? count : capacity;
      }
      // one status update per warp
      const int cmax = __reduce_max_sync(0xffffffffu, act ? count : 0);
      if (lane == 0) {
        atomicMax(&status[ST_MAXNEIGH], cmax);
        if (cmax > capacity) atomicExch(&status[ST_OVERFLOW], 1);
      }
    }
    return;
  }
  // fallback (a tile or a cell too crowded for shared memory): one thread
  // per owned atom, candidates read from global memory, FP64 test
  for (int i = a0 + lane; i < a1; i += 32) {
    const double4 xi = x4[i];
    const int ti = (int)xi.w;
    int count = 0;
    int4 buf = make_int4(0, 0, 0, 0);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int id = (warp + 1 + dx) + (kTileCells + 2) * ((1 + dy) + 3 * (1 + dz));
          const int code = md_code(dx, dy, dz);
          const int g = s_src[id];
          const int j1 = cell_start[g + 1];
          for (int j = cell_start[g]; j < j1; j++) {
            if (code == MD_CODE_SELF && j == i) continue;
            const double4 xj = x4[j];
            if (exact_pair(xi, xj, s_sh[id][0], s_sh[id][1], s_sh[id][2],
                           cns[ti * ntp1 + (int)xj.w]))
              append_entry(nlist, stride, i, count, capacity, md_make_entry(j, code), buf);
          }
        }
    flush_entries(nlist, stride, i, count, capacity, buf);
    numneigh[i] = count < capacity ? count : capacity;
    atomicMax(&status[ST_MAXNEIGH], count);
    if (count > capacity) atomicExch(&status[ST_OVERFLOW], 1);
  }
}

// ---------------------------------------------------------------------------
// Export of Neighbor::half_bin_newton's half list from the full list.
struct HalfBins {
  double lo[3], hi[3], bininv[3], binsize[3];
  int nbin[3], mbinlo[3];
  int sx, sy, sz;
  double cutneighmaxsq;
};

__device__ __forceinline__ int coord2bin_dim(double x, double lo, double hi, double inv, int nbin) {
  // Neighbor::coord2bin for one dimension (src/neighbor.cpp:1918-1947)
  int ix;
  if (x >= hi) ix = (int)((x - hi) * inv) + nbin;
  else if (x >= lo) {
    ix = (int)((x - lo) * inv);
    ix = ix < nbin - 1 ? ix : nbin - 1;
  } else ix = (int)((x - lo) * inv) - 1;
  return ix;
}

__device__ __forceinline__ double bin_distance(const HalfBins &b, int i, int j, int k) {
  double dx = i > 0 ? (i - 1) * b.binsize[0] : (i == 0 ? 0.0 : (i + 1) * b.binsize[0]);
  double dy = j > 0 ? (j - 1) * b.binsize[1] : (j == 0 ? 0.0 : (j + 1) * b.binsize[1]);
  double dz = k > 0 ? (k - 1) * b.binsize[2] : (k == 0 ? 0.0 : (k + 1) * b.binsize[2]);
  return dx * dx + dy * dy + dz * dz;
}

template <bool WRITE>
__global__ void k_half(int n, int stride, BoxGeom box, HalfBins hb, const double4 *__restrict__ x4,
                       const int *__restrict__ cell, const int *__restrict__ orig,
                       const int *__restrict__ nlist, const int *__restrict__ numneigh,
                       int *__restrict__ count_out, const long long *__restrict__ offset,
                       int *__restrict__ jowner, int *__restrict__ jimage, long long cap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 xi = x4[i];
  int bi[3] = {coord2bin_dim(xi.x, hb.lo[0], hb.hi[0], hb.bininv[0], hb.nbin[0]),
               coord2bin_dim(xi.y, hb.lo[1], hb.hi[1], hb.bininv[1], hb.nbin[1]),
               coord2bin_dim(xi.z, hb.lo[2], hb.hi[2], hb.bininv[2], hb.nbin[2])};
  int cx, cy, cz;
  md_cell_unpack(cell[i], cx, cy, cz);
  int ci[3] = {cx, cy, cz};
  int oi = orig[i];
  int num = numneigh[i];
  long long out = WRITE ? offset[oi] : 0;
  int cnt = 0;
  for (int k = 0; k < num; k++) {
    unsigned int e = (unsigned int)nlist[md_slab(k, i, stride)];
    int j, dc[3];
    md_entry(e, j, dc[0], dc[1], dc[2]);
    int s[3];
    double g[3];
    double4 xj = x4[j];
    double xjv[3] = {xj.x, xj.y, xj.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      int c = ci[d] + dc[d];
      s[d] = c < 0 ? -1 : (c >= box.ncell[d] ? 1 : 0);
      g[d] = __dadd_rn(xjv[d], s[d] * box.prd[d]);
    }
    int bj[3] = {coord2bin_dim(g[0], hb.lo[0], hb.hi[0], hb.bininv[0], hb.nbin[0]),
                 coord2bin_dim(g[1], hb.lo[1], hb.hi[1], hb.bininv[1], hb.nbin[1]),
                 coord2bin_dim(g[2], hb.lo[2], hb.hi[2], hb.bininv[2], hb.nbin[2])};
    int ox = bj[0] - bi[0], oy = bj[1] - bi[1], oz = bj[2] - bi[2];
    bool ghost = (s[0] | s[1] | s[2]) != 0;
    bool own;
    if (ox == 0 && oy == 0 && oz == 0) {
      if (!ghost) own = orig[j] > oi;  // j beyond i in the bin's linked list
      else {                            // ghost "above and to the right"
        own = !(g[2] < xi.z) &&
              !(g[2] == xi.z && (g[1] < xi.y || (g[1] == xi.y && g[0] < xi.x)));
      }
    } else {
      own = (oz > 0 || oy > 0 || (oy == 0 && ox > 0)) && oz >= 0 && oz <= hb.sz &&
            ox >= -hb.sx && ox <= hb.sx && oy >= -hb.sy && oy <= hb.sy &&
            bin_distance(hb, ox, oy, oz) < hb.cutneighmaxsq;
    }
    if (own) {
      if (WRITE && out + cnt < cap) {
        jowner[out + cnt] = orig[j];
        jimage[out + cnt] = (s[0] + 1) + 3 * (s[1] + 1) + 9 * (s[2] + 1);
      }
      cnt++;
    }
  }
  if (!WRITE) count_out[oi] = cnt;
}

__global__ void k_prefix_ll(int n, const int *__restrict__ cnt, long long *__restrict__ off,
                            long long *__restrict__ total) {
  // single-thread prefix over atoms (export path only, not per step)
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  long long s = 0;
  for (int i = 0; i < n; i++) {
    off[i] = s;
    s += cnt[i];
  }
  *total = s;
}

}  // namespace

// Staging capacity of a builder tile: 1.25 x the atoms of kStageCells cells
// at the densest replica's mean count per cell, or the most any tile staged
// in an earlier build if that is larger, rounded up to 128 and at most
// kStageCapMax.  A tile that stages more atoms takes the global-memory path
// (same list, slower); a smaller capacity leaves room for more resident
// CTAs per SM.
static int round_cap(int cap) {
  cap = (cap + 127) & ~127;
  if (cap < 256) cap = 256;
  return cap < kStageCapMax ? cap : kStageCapMax;
}

// Staging capacity of the builder tiles: 1.25 x the mean atom count of the 54
// staged cells, raised when a build reports a more crowded tile.  For a batch
// the mean is the batch's (the common case, at full occupancy); the densest
// replicas' tiles are rebuilt in a second pass with md_stage_cap2.
int md_stage_cap(const b200_ctx *c) {
  const double per_cell = c->ncells > 0 ? (double)c->n / c->ncells : 0.0;
  int cap = (int)(1.25 * kStageCells * per_cell) + 64;
  if (!c->nrep && c->stage_need > cap) cap = c->stage_need;
  return round_cap(cap);
}

// second-pass capacity of a batch: the densest replica's tiles (0 when the
// first pass holds every tile)
int md_stage_cap2(const b200_ctx *c) {
  if (!c->nrep) return 0;
  double per_cell = 0.0;
  for (int r = 0; r < c->nrep; r++) {
    const BoxGeom &b = c->rep_box[r];
    const double d = (double)c->rep_natoms[r] / ((double)b.ncell[0] * b.ncell[1] * b.ncell[2]);
    per_cell = d > per_cell ? d : per_cell;
  }
  int cap = (int)(1.25 * kStageCells * per_cell) + 64;
  if (c->stage_need > cap) cap = c->stage_need;
  cap = round_cap(cap);
  return cap > md_stage_cap(c) ? cap : 0;
}

// After a build: raise the staging capacity when some tile staged more atoms
// than the current one holds.  Returns true when the capacity changed (the
// caller re-captures its graphs).
bool md_stage_feedback(b200_ctx *c, int staged_max) {
  const int cap = c->nrep ? (md_stage_cap2(c) > 0 ? md_stage_cap2(c) : md_stage_cap(c))
                          : md_stage_cap(c);
  if (staged_max <= cap || cap >= kStageCapMax) return false;
  c->stage_need = staged_max + staged_max / 10;
  const int now = c->nrep ? (md_stage_cap2(c) > 0 ? md_stage_cap2(c) : md_stage_cap(c))
                          : md_stage_cap(c);
  return now != cap;
}

static cudaError_t launch_scan(b200_ctx *c, int m, const int *in, int *out, const int *flag) {
  int tiles = (m + kScanTile - 1) / kScanTile;
  if (tiles > kScanTile) return cudaErrorInvalidValue;
  int *sums = c->scan_tmp;
  k_scan_tiles<<<tiles, kScanThreads, 0, c->stream>>>(m, in, out, sums, flag);
  c->launches++;
  if (tiles > 1) {
    k_scan_tiles<<<1, kScanThreads, 0, c->stream>>>(tiles, sums, sums, nullptr, flag);
    k_scan_add<<<tiles, 256, 0, c->stream>>>(m, out, sums, flag);
    c->launches += 2;
  }
  return cudaGetLastError();
}

cudaError_t md_rebuild(b200_ctx *c, const int *d_flag) {
  const int n = c->n, B = 256;
  const int m = c->ncells + 1;
  const Reps R = c->reps();
  if (c->nrep)
    k_wrap_bin<true><<<md_blocks(n, B), B, 0, c->stream>>>(n, c->box, R, c->x4, c->image,
                                                           c->cell_count, c->slot, c->cell_tmp,
                                                           c->status, d_flag);
  else
    k_wrap_bin<false><<<md_blocks(n, B), B, 0, c->stream>>>(n, c->box, R, c->x4, c->image,
                                                            c->cell_count, c->slot, c->cell_tmp,
                                                            c->status, d_flag);
  c->launches += 1;
  cudaError_t e = launch_scan(c, m, c->cell_count, c->cell_start, d_flag);
  if (e != cudaSuccess) return e;
  k_scatter<<<md_blocks(n, B), B, 0, c->stream>>>(n, c->cell_tmp, c->slot, c->cell_start, c->perm,
                                                  m, c->cell_count, d_flag);
  k_sort_cells<<<md_blocks(c->ncells, kSortWarps), kSortWarps * 32, 0, c->stream>>>(
      c->ncells, c->cell_start, c->perm, c->slot, c->orig, d_flag);
  if (c->nrep)
    k_gather<true><<<md_blocks(n, B), B, 0, c->stream>>>(
        n, c->stride, c->box, R, c->perm, c->x4, c->x4b, c->v, c->vb, c->orig, c->origb, c->image,
        c->imageb, c->cell_tmp, c->cell, c->prec == 1 ? c->xq : nullptr,
        c->check ? c->xhold : nullptr, d_flag);
  else
    k_gather<false><<<md_blocks(n, B), B, 0, c->stream>>>(
        n, c->stride, c->box, R, c->perm, c->x4, c->x4b, c->v, c->vb, c->orig, c->origb, c->image,
        c->imageb, c->cell_tmp, c->cell, c->prec == 1 ? c->xq : nullptr,
        c->check ? c->xhold : nullptr, d_flag);
  k_copyback<<<md_blocks(n, B), B, 0, c->stream>>>(n, c->stride, c->x4b, c->x4, c->vb, c->v,
                                                   c->origb, c->orig, c->imageb, c->image,
                                                   c->where, c->status, d_flag);
  {
    const int tiles = c->nrep ? c->ntiles
                              : ((c->box.ncell[0] + kTileCells - 1) / kTileCells) *
                                    c->box.ncell[1] * c->box.ncell[2];
    // the shared-memory opt-in, once per device this process uses
    static unsigned long long smem_opt_in = 0ull;
    const unsigned long long dev_bit = 1ull << (c->device & 63);
    if (!(smem_opt_in & dev_bit)) {
      const int most = (int)neigh_smem(kStageCapMax);
      cudaFuncSetAttribute(k_neigh_tiles<true, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, most);
      cudaFuncSetAttribute(k_neigh_tiles<true, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, most);
      cudaFuncSetAttribute(k_neigh_tiles<false, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, most);
      cudaFuncSetAttribute(k_neigh_tiles<false, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, most);
      smem_opt_in |= dev_bit;
    }
    const int cap = md_stage_cap(c);
    const int cap2 = md_stage_cap2(c);  // a batch's densest tiles, or 0
    auto launch = [&](int stage_cap, int pass, cudaStream_t st) {
      const size_t smem = neigh_smem(stage_cap);
#define MD_NEIGH_ARGS                                                                         \
  n, c->stride, c->capacity, stage_cap, c->box, R, c->ntypes + 1, c->cutneighsq_dev, c->x4,  \
      c->cell_start, c->nlist, c->numneigh, c->status, d_flag, pass, cap
      if (c->ntypes == 1 && !c->nrep)
        k_neigh_tiles<true, false><<<tiles, kNeighThreads, smem, st>>>(MD_NEIGH_ARGS);
      else if (c->ntypes == 1)
        k_neigh_tiles<true, true><<<tiles, kNeighThreads, smem, st>>>(MD_NEIGH_ARGS);
      else if (!c->nrep)
        k_neigh_tiles<false, false><<<tiles, kNeighThreads, smem, st>>>(MD_NEIGH_ARGS);
      else
        k_neigh_tiles<false, true><<<tiles, kNeighThreads, smem, st>>>(MD_NEIGH_ARGS);
#undef MD_NEIGH_ARGS
      c->launches++;
    };
    if (cap2 > 0) {
      // The two passes build disjoint tiles, so the second (the densest
      // tiles, large staging, few blocks per SM) runs on the side stream
      // beside the first instead of after it; the join makes the main stream
      // wait for both.  Inside a graph capture the fork and join become
      // graph dependencies.
      cudaError_t e = cudaEventRecord(c->ev_fork, c->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_aux, c->ev_fork, 0);
      if (e != cudaSuccess) return e;
      launch(cap, 1, c->stream);
      launch(cap2, 2, c->s_aux);
      e = cudaEventRecord(c->ev_join, c->s_aux);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_join, 0);
      if (e != cudaSuccess) return e;
    } else {
      launch(cap, 0, c->stream);
    }
  }
  c->launches += 3;
  return cudaGetLastError();
}

// LAMMPS bins of Neighbor::setup_bins (src/neighbor.cpp:1538-1702) for a
// single periodic process: binsize = cutneighmax/2, bounding box extended by
// the ghost cutoff, half stencil extents sx, sy, sz.
static HalfBins half_bins(const b200_ctx *c) {
  HalfBins hb{};
  const double SMALL = 1.0e-6;
  double cutghost = c->cutneighmax;
  double binsize_optimal = 0.5 * c->cutneighmax;
  double bbox[3];
  for (int d = 0; d < 3; d++) bbox[d] = c->box.hi[d] - c->box.lo[d];
  if (binsize_optimal == 0.0) binsize_optimal = bbox[0];
  double binsizeinv = 1.0 / binsize_optimal;
  for (int d = 0; d < 3; d++) {
    hb.lo[d] = c->box.lo[d];
    hb.hi[d] = c->box.hi[d];
    int nb = (int)(bbox[d] * binsizeinv);
    if (nb == 0) nb = 1;
    hb.nbin[d] = nb;
    hb.binsize[d] = bbox[d] / nb;
    hb.bininv[d] = 1.0 / hb.binsize[d];
    double coord = (c->box.lo[d] - cutghost) - SMALL * bbox[d];
    int lo = (int)((coord - c->box.lo[d]) * hb.bininv[d]);
    if (coord < c->box.lo[d]) lo = lo - 1;
    hb.mbinlo[d] = lo - 1;
  }
  int s[3];
  for (int d = 0; d < 3; d++) {
    s[d] = (int)(c->cutneighmax * hb.bininv[d]);
    if (s[d] * hb.binsize[d] < c->cutneighmax) s[d]++;
  }
  hb.sx = s[0];
  hb.sy = s[1];
  hb.sz = s[2];
  hb.cutneighmaxsq = c->cutneighmax * c->cutneighmax;
  return hb;
}

cudaError_t md_half_list(b200_ctx *c, int *d_num, int *d_jowner, int *d_jimage, long long cap,
                         long long *total) {
  const int n = c->n, B = 128;
  HalfBins hb = half_bins(c);
  long long *d_off = nullptr, *d_total = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&d_off, sizeof(long long) * (size_t)(n + 1), c->stream);
  if (e != cudaSuccess) return e;
  e = cudaMallocAsync((void **)&d_total, sizeof(long long), c->stream);
  if (e != cudaSuccess) return e;
  k_half<false><<<md_blocks(n, B), B, 0, c->stream>>>(n, c->stride, c->box, hb, c->x4, c->cell,
                                                      c->orig, c->nlist, c->numneigh, d_num,
                                                      nullptr, nullptr, nullptr, 0);
  k_prefix_ll<<<1, 1, 0, c->stream>>>(n, d_num, d_off, d_total);
  if (d_jowner && cap > 0)
    k_half<true><<<md_blocks(n, B), B, 0, c->stream>>>(n, c->stride, c->box, hb, c->x4, c->cell,
                                                       c->orig, c->nlist, c->numneigh, nullptr,
                                                       d_off, d_jowner, d_jimage, cap);
  c->launches += d_jowner && cap > 0 ? 3 : 2;
  e = cudaMemcpyAsync(total, d_total, sizeof(long long), cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return e;
  cudaFreeAsync(d_off, c->stream);
  cudaFreeAsync(d_total, c->stream);
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}
