/* ----------------------------------------------------------------------
   run_style verlet/b200 -- the Verlet loop on the GPU for systems the
   device path covers.
------------------------------------------------------------------------- */

#include <cstring>

#include "b200_link.h"
#include "b200md.h"
#include "dump_custom_b200.h"
#include "fix_nve_b200.h"
#include "verlet_b200.h"

#include "atom.h"
#include "error.h"
#include "fix.h"
#include "force.h"
#include "group.h"
#include "modify.h"
#include "neighbor.h"
#include "output.h"
#include "pair.h"
#include "thermo.h"
#include "timer.h"
#include "update.h"

using namespace LAMMPS_NS;

VerletB200::VerletB200(LAMMPS *lmp, int narg, char **arg) : Verlet(lmp, narg, arg) {
  link = B200Link::instance(lmp);
  tables = NULL;
  resident = 0;
  ncalls0 = ndanger0 = 0;
}

VerletB200::~VerletB200() { B200Link::release(lmp); }

void VerletB200::init() {
  Verlet::init();
  tables = force->pair ? dynamic_cast<B200PairTables *>(force->pair) : NULL;
  resident = tables != NULL;
  if (atom->molecular || force->kspace || atom->rmass_flag) resident = 0;
  // by class: a fix created through the -sf b200 suffix keeps the style
  // name it was given ("nve"), src/modify.cpp:715-727 and src/fix.cpp:46-47
  if (modify->nfix != 1 || !dynamic_cast<FixNVEB200 *>(modify->fix[0]) ||
      modify->fix[0]->igroup != 0)
    resident = 0;
  if (modify->n_post_integrate || modify->n_pre_exchange || modify->n_pre_neighbor ||
      modify->n_pre_force || modify->n_post_force || modify->n_end_of_step)
    resident = 0;
  if (resident) {
    link->check_supported("run_style verlet/b200");
    link->banner("B200: run_style verlet/b200 (VerletB200), resident mode: the run advances "
                 "on the device");
  } else {
    link->banner("B200: run_style verlet/b200 (VerletB200), per-call mode: Verlet::run with "
                 "the /b200 pair style");
  }
}

/* Verlet::setup (forces at the current step through the per-call pair
   path, step-0 output), then the full state goes to the device, whose own
   b200_setup recomputes the same forces */
void VerletB200::setup() {
  Verlet::setup();
  if (!resident) return;
  link->sync_settings(tables);
  link->upload_atoms(1);
  link->reset_images();
  double row[9];
  link->check(b200_setup(link->ctx, row), "setup");
  ncalls0 = neighbor->ncalls;
  ndanger0 = neighbor->ndanger;
}

void VerletB200::run(int n) {
  if (!resident) {
    Verlet::run(n);
    return;
  }
  b200_ctx *ctx = link->ctx;
  const bigint end = update->ntimestep + n;
  while (update->ntimestep < end) {
    // advance on the device to the next output step (or the end of the run)
    bigint stop = output->next < end ? output->next : end;
    if (stop <= update->ntimestep) stop = update->ntimestep + 1;
    const int k = (int)(stop - update->ntimestep);
    double row[9];
    int nrows = 0;
    timer->stamp();
    link->check(b200_run(ctx, k, update->dt, force->ftm2v, 0, row, 1, &nrows), "run");
    timer->stamp(TIME_PAIR);
    update->ntimestep = stop;

    // host arrays and the pair's tallies for this step's output: at the end
    // of the run all of them; on an output step, the velocities that the
    // default thermo reads (Temp, Press), and the rest only when an output
    // other than `dump custom/b200` is due (which gathers its own columns)
    if (stop == end || !output_needs_velocities_only(stop)) {
      link->download_state();
    } else {
      link->stale = B200_FIELD_X | B200_FIELD_V | B200_FIELD_F | B200_FIELD_IMAGE;
      link->refresh(B200_FIELD_V);
      long long total = 0;
      int nc = 0, nd = 0, maxneigh = 0, cap = 0;
      link->check(b200_neigh_stats(ctx, &total, &nc, &nd, &maxneigh, &cap), "stats");
      if (maxneigh > neighbor->oneatom) link->check(B200_ERR_NEIGH_OVERFLOW, "run");
    }
    ev_set(stop);
    Pair *pair = force->pair;
    if (nrows > 0) {
      pair->eng_vdwl = row[2];
      pair->eng_coul = 0.0;
      for (int m = 0; m < 6; m++) pair->virial[m] = row[3 + m];
    }
    long long total = 0;
    int ncalls = 0, ndanger = 0, maxneigh = 0, cap = 0;
    link->check(b200_neigh_stats(ctx, &total, &ncalls, &ndanger, &maxneigh, &cap), "stats");
    neighbor->ncalls = ncalls0 + ncalls;
    neighbor->ndanger = ndanger0 + ndanger;
    if (stop == output->next) {
      timer->stamp();
      output->write(stop);
      timer->stamp(TIME_OUTPUT);
    }
  }
}

/* true when the output due at `step` is the default thermo line (which reads
   velocities, plus the pair's energy and virial taken from the device's
   thermo row) and dumps of style custom/b200 only */
int VerletB200::output_needs_velocities_only(bigint step) {
  if (step != output->next) return 1;  // no output: the host is not read
  if (output->restart_flag && output->next_restart == step) return 0;
  if (output->next_thermo == step && strcmp(output->thermo->style, "one") != 0) return 0;
  for (int i = 0; i < output->ndump; i++)
    if (output->next_dump[i] == step && !dynamic_cast<DumpCustomB200 *>(output->dump[i]))
      return 0;
  return 1;
}
