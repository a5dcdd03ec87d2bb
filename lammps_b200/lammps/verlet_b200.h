/* -*- c++ -*- ----------------------------------------------------------
   run_style verlet/b200

   Verlet (src/verlet.h) whose run(n) advances the atoms on the GPU when the
   system is one the device path covers: a /b200 pair style, `fix nve/b200`
   on group all as the only fix, no bonds, no kspace.  Atoms stay on the
   device between output steps; on each output step the positions,
   velocities, forces and image flags are copied back, the pair's energy and
   virial are set from the device's thermo row, and Output::write runs as
   usual.  Any other system runs the plain Verlet loop, with /b200 pair
   styles computing forces per call.
------------------------------------------------------------------------- */

#ifdef INTEGRATE_CLASS

IntegrateStyle(verlet/b200,VerletB200)

#else

#ifndef LMP_VERLET_B200_H
#define LMP_VERLET_B200_H

#include "verlet.h"

namespace LAMMPS_NS {

class VerletB200 : public Verlet {
 public:
  VerletB200(class LAMMPS *, int, char **);
  virtual ~VerletB200();
  void init();
  void setup();
  void run(int);

 private:
  class B200Link *link;
  class B200PairTables *tables;
  int resident;
  bigint ncalls0, ndanger0;  // host neighbor counters at setup
  int output_needs_velocities_only(bigint step);
};

}

#endif
#endif
