/* ----------------------------------------------------------------------
   fix nve/b200 -- FixNVE whose half-steps move to the device under
   run_style verlet/b200.
------------------------------------------------------------------------- */

#include "fix_nve_b200.h"

#include "atom.h"
#include "error.h"

using namespace LAMMPS_NS;

FixNVEB200::FixNVEB200(LAMMPS *lmp, int narg, char **arg) : FixNVE(lmp, narg, arg) {}

void FixNVEB200::init() {
  FixNVE::init();
  // the device integrator uses per-type masses (FixNVE's mass[type] branch,
  // src/fix_nve.cpp:91-104)
  if (atom->rmass_flag) error->all(FLERR, "fix nve/b200 requires per-type masses");
}
