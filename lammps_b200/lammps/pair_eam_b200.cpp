/* ----------------------------------------------------------------------
   pair_style eam/b200 (and eam/alloy/b200, eam/fs/b200) -- PairEAM
   evaluated by libb200md.
------------------------------------------------------------------------- */

#include <cstdio>
#include <cstring>

#include "b200md.h"
#include "pair_eam_b200.h"

#include "atom.h"
#include "error.h"

using namespace LAMMPS_NS;

PairEAMB200::PairEAMB200(LAMMPS *lmp) : PairEAM(lmp) {
  precision = B200_PREC_FP64;
  no_virial_fdotr_compute = 1;
  link = B200Link::instance(lmp);
}

PairEAMB200::~PairEAMB200() { B200Link::release(lmp); }

PairEAMAlloyB200::PairEAMAlloyB200(LAMMPS *lmp)
    : PairEAM(lmp), PairEAMB200(lmp), PairEAMAlloy(lmp) {}

PairEAMFSB200::PairEAMFSB200(LAMMPS *lmp) : PairEAM(lmp), PairEAMB200(lmp), PairEAMFS(lmp) {}

/* pair_style eam takes no arguments (src/MANYBODY/pair_eam.cpp:318-321);
   the /b200 forms accept `precision fp64|mixed` */
void PairEAMB200::settings(int narg, char **arg) {
  if (narg == 0) return;
  if (narg != 2 || strcmp(arg[0], "precision") != 0) error->all(FLERR, "Illegal pair_style command");
  if (strcmp(arg[1], "fp64") == 0) precision = B200_PREC_FP64;
  else if (strcmp(arg[1], "mixed") == 0) precision = B200_PREC_MIXED;
  else error->all(FLERR, "Illegal pair_style command");
}

/* PairEAM::init_style (src/MANYBODY/pair_eam.cpp:397-405) without the
   NeighList request: the device builds its own list */
void PairEAMB200::init_style() {
  link->check_supported("pair_style eam/b200");
  file2array();
  array2spline();
  link->tables_dirty = 1;
  char msg[160];
  snprintf(msg, sizeof(msg), "B200: pair_style %s (%s), device neighbor list", b200_style(),
           b200_class());
  link->banner(msg);
}

double PairEAMB200::init_one(int i, int j) {
  link->tables_dirty = 1;
  return PairEAM::init_one(i, j);
}

/* the 7-coefficient splines of array2spline, row 0 unused, and the type maps
   of file2array, passed straight through (layouts of include/b200md.h) */
int PairEAMB200::b200_upload_tables(b200_ctx *ctx) {
  return b200_set_eam(ctx, atom->ntypes, nrho, drho, nr, dr, rhomax, cutmax, nfrho,
                      &frho_spline[0][0][0], nrhor, &rhor_spline[0][0][0], nz2r,
                      &z2r_spline[0][0][0], type2frho, &type2rhor[0][0], &type2z2r[0][0]);
}

void PairEAMB200::compute(int eflag, int vflag) {
  if (eflag || vflag) ev_setup(eflag, vflag);
  else evflag = vflag_fdotr = 0;
  link->pair_compute(this, this, eflag, vflag);
}
