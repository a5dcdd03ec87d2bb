/* ----------------------------------------------------------------------
   pair_style lj/cut/b200 -- PairLJCut evaluated by libb200md.
------------------------------------------------------------------------- */

#include <cstring>
#include <vector>

#include "b200md.h"
#include "pair_lj_cut_b200.h"

#include "atom.h"
#include "error.h"
#include "force.h"
#include "neighbor.h"
#include "update.h"

using namespace LAMMPS_NS;

PairLJCutB200::PairLJCutB200(LAMMPS *lmp) : PairLJCut(lmp) {
  precision = B200_PREC_FP64;
  // the device computes the pairwise virial itself (full list, no ghosts)
  no_virial_fdotr_compute = 1;
  link = B200Link::instance(lmp);
}

PairLJCutB200::~PairLJCutB200() { B200Link::release(lmp); }

/* trailing `precision fp64|mixed` keyword, the rest as PairLJCut::settings */
void PairLJCutB200::settings(int narg, char **arg) {
  if (narg >= 3 && strcmp(arg[narg - 2], "precision") == 0) {
    if (strcmp(arg[narg - 1], "fp64") == 0) precision = B200_PREC_FP64;
    else if (strcmp(arg[narg - 1], "mixed") == 0) precision = B200_PREC_MIXED;
    else error->all(FLERR, "Illegal pair_style command");
    narg -= 2;
  }
  PairLJCut::settings(narg, arg);
}

/* the device builds its own list: no NeighList request (the GPU package's
   device-neighbor mode, src/GPU/pair_lj_cut_gpu.cpp:161-165) */
void PairLJCutB200::init_style() {
  link->check_supported("pair_style lj/cut/b200");
  // PairLJCut::init_style (src/pair_lj_cut.cpp:519-526) is where cut_respa
  // is set, and PairLJCut::init_one reads it; the device has no rRESPA levels
  if (strstr(update->integrate_style, "respa"))
    error->all(FLERR, "pair_style lj/cut/b200 does not support run_style respa");
  cut_respa = NULL;
  link->tables_dirty = 1;
  link->banner("B200: pair_style lj/cut/b200 (PairLJCutB200), device neighbor list");
}

double PairLJCutB200::init_one(int i, int j) {
  link->tables_dirty = 1;
  return PairLJCut::init_one(i, j);
}

/* cutsq, lj1..lj4, offset after init_one (src/pair_lj_cut.cpp:545-602) as
   (ntypes+1)^2 row-major tables */
int PairLJCutB200::b200_upload_tables(b200_ctx *ctx) {
  const int nt = atom->ntypes, w = nt + 1;
  std::vector<double> t(6 * w * w, 0.0);
  double *cs = &t[0], *l1 = cs + w * w, *l2 = l1 + w * w, *l3 = l2 + w * w, *l4 = l3 + w * w,
         *of = l4 + w * w;
  for (int i = 1; i <= nt; i++)
    for (int j = 1; j <= nt; j++) {
      const int k = i * w + j;
      cs[k] = cutsq[i][j];
      l1[k] = lj1[i][j];
      l2[k] = lj2[i][j];
      l3[k] = lj3[i][j];
      l4[k] = lj4[i][j];
      of[k] = offset[i][j];
    }
  return b200_set_lj(ctx, nt, cs, l1, l2, l3, l4, of);
}

void PairLJCutB200::compute(int eflag, int vflag) {
  if (eflag || vflag) ev_setup(eflag, vflag);
  else evflag = vflag_fdotr = 0;
  link->pair_compute(this, this, eflag, vflag);
}
