// integrate.cu -- velocity-Verlet (fix nve), the kinetic-energy reduction,
// the device-side rebuild decision and thermo-row recording.
//
// FixNVE::initial_integrate / final_integrate (src/fix_nve.cpp:65-142) with
// dtfm = dtf / mass[type]; every product and sum is rounded separately as in
// the reference.  The initial half-kick also refreshes the fixed-point
// coordinates used by the mixed-precision pair kernels (md_xq) and flags any
// atom that moved more than half the skin since the last build
// (Neighbor::check_distance, src/neighbor.cpp:1322-1372).
#include "md_state.h"

namespace {

__global__ void k_decide(int *status, int every, int delay, int check, int *dcount, int *mail) {
  md_decide_dev(status, every, delay, check, dcount, mail);
}

__global__ void k_record_row(int *status, const double *ev, double *rows, int cap) {
  md_record_row_dev(status, ev, rows, cap);
}

template <bool BATCH>
__global__ void __launch_bounds__(256) k_nve_initial(int n, int stride, double dtv, double dtf,
                                                      const double *__restrict__ mass,
                                                      double4 *__restrict__ x4,
                                                      double *__restrict__ v,
                                                      const double *__restrict__ f,
                                                      int4 *__restrict__ xq, BoxGeom box1,
                                                      Reps reps,
                                                      const double4 *__restrict__ xhold,
                                                      double triggersq, int *__restrict__ status,
                                                      const int *__restrict__ ghost,
                                                      const int *__restrict__ orig) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool moved = false;
  // a ghost (an atom another rank owns) is neither moved nor checked here:
  // the halo unpack overwrites its position with the owner's
  if (i < n && !(ghost && ghost[orig[i]])) {
    double4 p = x4[i];
    const double dtfm = dtf / mass[(int)p.w];
    double vx = __dadd_rn(v[i], __dmul_rn(dtfm, f[i]));
    double vy = __dadd_rn(v[stride + i], __dmul_rn(dtfm, f[stride + i]));
    double vz = __dadd_rn(v[2 * stride + i], __dmul_rn(dtfm, f[2 * stride + i]));
    p.x = __dadd_rn(p.x, __dmul_rn(dtv, vx));
    p.y = __dadd_rn(p.y, __dmul_rn(dtv, vy));
    p.z = __dadd_rn(p.z, __dmul_rn(dtv, vz));
    v[i] = vx;
    v[stride + i] = vy;
    v[2 * stride + i] = vz;
    x4[i] = p;
    if (xq) xq[i] = md_xq(p, BATCH ? reps.box[reps.rep_of_atom[i]] : box1);
    if (xhold) {
      const double4 h = xhold[i];
      const double rsq = dsq3(__dsub_rn(p.x, h.x), __dsub_rn(p.y, h.y), __dsub_rn(p.z, h.z));
      moved = rsq > triggersq;
    }
  }
  if (xhold && __any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0)
    atomicExch(&status[ST_MOVED], 1);
}

template <bool KE>
__global__ void __launch_bounds__(256) k_nve_final(int n, int stride, double dtf,
                                                    const double *__restrict__ mass,
                                                    const double4 *__restrict__ x4,
                                                    double *__restrict__ v,
                                                    const double *__restrict__ f,
                                                    double *partial, unsigned int *counter,
                                                    double *out, const int *__restrict__ ghost,
                                                    const int *__restrict__ orig) {
  __shared__ double red[8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < n && !(ghost && ghost[orig[i]])) {
    const double m = mass[(int)x4[i].w];
    const double dtfm = dtf / m;
    const double vx = __dadd_rn(v[i], __dmul_rn(dtfm, f[i]));
    const double vy = __dadd_rn(v[stride + i], __dmul_rn(dtfm, f[stride + i]));
    const double vz = __dadd_rn(v[2 * stride + i], __dmul_rn(dtfm, f[2 * stride + i]));
    v[i] = vx;
    v[stride + i] = vy;
    v[2 * stride + i] = vz;
    // ComputeTemp::compute_scalar term (src/compute_temp.cpp:84-86)
    if (KE) acc[0] = (vx * vx + vy * vy + vz * vz) * m;
  }
  if (KE) block_partials_finish<1>(acc, red, partial, counter, out, false);
}

// FixNVE::final_integrate of this step, the kinetic-energy term of the
// thermo output (KE), then FixNVE::initial_integrate of the next step: the
// same rounded operations as k_nve_final followed by k_nve_initial, with v, f
// and x read once.  The last block to finish then completes the step on the
// device: the kinetic-energy sum (block partials added in block order), the
// thermo row (KE), and the next step's rebuild decision (Neighbor::decide),
// which sees every block's displacement flag.
template <bool KE, bool BATCH>
__global__ void __launch_bounds__(256) k_nve_fused(int n, int stride, double dtv, double dtf,
                                                    const double *__restrict__ mass,
                                                    double4 *__restrict__ x4,
                                                    double *__restrict__ v,
                                                    const double *__restrict__ f,
                                                    int4 *__restrict__ xq, BoxGeom box1,
                                                    Reps reps, const double4 *__restrict__ xhold,
                                                    double triggersq, int *__restrict__ status,
                                                    double *partial, unsigned int *counter,
                                                    double *ev, double *rows, int rows_cap,
                                                    int every, int delay, int check, int *dcount,
                                                    int *mail) {
  __shared__ double red[8];
  __shared__ bool last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  bool moved = false;
  if (i < n) {
    const BoxGeom &box = BATCH ? reps.box[reps.rep_of_atom[i]] : box1;
    moved = md_nve_fused_atom<KE>(i, stride, dtv, dtf, mass, x4, v, f, xq, box, xhold,
                                  triggersq, acc[0]);
  }
  if (xhold && __any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) {
    atomicExch(&status[ST_MOVED], 1);
    __threadfence();  // the flag is visible before this block counts itself done
  }
  if (KE) block_sum<1>(acc, red);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (KE) partial[blockIdx.x] = acc[0];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (KE) {
    double s[1] = {0.0};
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s[0] += __ldcg(&partial[b]);
    __syncthreads();
    block_sum<1>(s, red);
    if (threadIdx.x == 0) ev[7] = s[0];
  }
  if (threadIdx.x == 0) {
    if (KE) md_record_row_dev(status, ev, rows, rows_cap);
    md_decide_dev(status, every, delay, check, dcount, mail);
    *counter = 0u;
  }
}

__global__ void __launch_bounds__(256) k_ke(int n, int stride, const double *__restrict__ mass,
                                             const double4 *__restrict__ x4,
                                             const double *__restrict__ v, double *partial,
                                             unsigned int *counter, double *out) {
  __shared__ double red[8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < n) {
    const double m = mass[(int)x4[i].w];
    const double vx = v[i], vy = v[stride + i], vz = v[2 * stride + i];
    acc[0] = (vx * vx + vy * vy + vz * vz) * m;
  }
  block_partials_finish<1>(acc, red, partial, counter, out, false);
}

}  // namespace

cudaError_t md_nve_initial(b200_ctx *c, double dtv, double dtf) {
  const int B = 256;
  const double triggersq = 0.25 * c->skin * c->skin;  // src/neighbor.cpp:239
  if (c->nrep)
    k_nve_initial<true><<<md_blocks(c->n, B), B, 0, c->stream>>>(
        c->n, c->stride, dtv, dtf, c->mass_dev, c->x4, c->v, c->f,
        c->prec == B200_PREC_MIXED ? c->xq : nullptr, c->box, c->reps(),
        c->check ? c->xhold : nullptr, triggersq, c->status, c->ghosts_on ? c->ghost : nullptr,
        c->orig);
  else
    k_nve_initial<false><<<md_blocks(c->n, B), B, 0, c->stream>>>(
        c->n, c->stride, dtv, dtf, c->mass_dev, c->x4, c->v, c->f,
        c->prec == B200_PREC_MIXED ? c->xq : nullptr, c->box, c->reps(),
        c->check ? c->xhold : nullptr, triggersq, c->status, c->ghosts_on ? c->ghost : nullptr,
        c->orig);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_nve_final(b200_ctx *c, double dtf, bool ke) {
  const int B = 256;
  const int *gh = c->ghosts_on ? c->ghost : nullptr;
  if (ke)
    k_nve_final<true><<<md_blocks(c->n, B), B, 0, c->stream>>>(
        c->n, c->stride, dtf, c->mass_dev, c->x4, c->v, c->f, c->partial, c->counter, c->ev + 7,
        gh, c->orig);
  else
    k_nve_final<false><<<md_blocks(c->n, B), B, 0, c->stream>>>(
        c->n, c->stride, dtf, c->mass_dev, c->x4, c->v, c->f, c->partial, c->counter, c->ev + 7,
        gh, c->orig);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_nve_fused(b200_ctx *c, double dtv, double dtf, bool ke) {
  const int B = 256;
  const double triggersq = 0.25 * c->skin * c->skin;  // src/neighbor.cpp:239
#define MD_FUSED_ARGS                                                                           \
  c->n, c->stride, dtv, dtf, c->mass_dev, c->x4, c->v, c->f,                                  \
      c->prec == B200_PREC_MIXED ? c->xq : nullptr, c->box, c->reps(),                        \
      c->check ? c->xhold : nullptr, triggersq, c->status, c->partial, c->counter, c->ev,     \
      c->rows, c->rows_cap, c->every, c->delay, c->check, c->dec_count, c->mail_dev
  const int grid = md_blocks(c->n, B);
  if (ke && c->nrep) k_nve_fused<true, true><<<grid, B, 0, c->stream>>>(MD_FUSED_ARGS);
  else if (ke) k_nve_fused<true, false><<<grid, B, 0, c->stream>>>(MD_FUSED_ARGS);
  else if (c->nrep) k_nve_fused<false, true><<<grid, B, 0, c->stream>>>(MD_FUSED_ARGS);
  else k_nve_fused<false, false><<<grid, B, 0, c->stream>>>(MD_FUSED_ARGS);
#undef MD_FUSED_ARGS
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_ke(b200_ctx *c) {
  const int B = 256;
  k_ke<<<md_blocks(c->n, B), B, 0, c->stream>>>(c->n, c->stride, c->mass_dev, c->x4, c->v,
                                                c->partial, c->counter, c->ev + 7);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_decide(b200_ctx *c) {
  k_decide<<<1, 1, 0, c->stream>>>(c->status, c->every, c->delay, c->check, c->dec_count,
                                   c->mail_dev);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_record_row(b200_ctx *c) {
  k_record_row<<<1, 1, 0, c->stream>>>(c->status, c->ev, c->rows, c->rows_cap);
  c->launches++;
  return cudaGetLastError();
}

cudaError_t md_zero_ev(b200_ctx *c) {
  return cudaMemsetAsync(c->ev, 0, 8 * sizeof(double), c->stream);
}
