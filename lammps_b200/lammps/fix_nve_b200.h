/* -*- c++ -*- ----------------------------------------------------------
   fix ID all nve/b200

   FixNVE (src/fix_nve.h).  Under the default run_style it integrates on the
   host exactly as fix nve does.  Under run_style verlet/b200 with a /b200
   pair style, the whole Verlet loop -- this fix's half-steps included --
   runs on the GPU (b200_run), and the host arrays are refreshed only on
   output steps.
------------------------------------------------------------------------- */

#ifdef FIX_CLASS

FixStyle(nve/b200,FixNVEB200)

#else

#ifndef LMP_FIX_NVE_B200_H
#define LMP_FIX_NVE_B200_H

#include "fix_nve.h"

namespace LAMMPS_NS {

class FixNVEB200 : public FixNVE {
 public:
  FixNVEB200(class LAMMPS *, int, char **);
  virtual ~FixNVEB200() {}
  void init();
};

}

#endif
#endif
