/* -*- c++ -*- ----------------------------------------------------------
   dump custom/b200 -- DumpCustom whose per-atom columns come straight from
   the device under run_style verlet/b200.

   Same arguments and output as `dump custom` (src/dump_custom.cpp).  In a
   resident run the host's x, v, f and image flags are behind the device
   between output steps; before DumpCustom::count() selects and packs the
   atoms, this style brings up to date only the groups its columns,
   thresholds and region read (positions, velocities, forces, image flags),
   gathered on the device (b200_gather) instead of downloading the whole
   state.  Columns it cannot trace to those groups (computes, fixes,
   variables, thresholds) refresh every group.
------------------------------------------------------------------------- */

#ifdef DUMP_CLASS

DumpStyle(custom/b200,DumpCustomB200)

#else

#ifndef LMP_DUMP_CUSTOM_B200_H
#define LMP_DUMP_CUSTOM_B200_H

#include "dump_custom.h"

namespace LAMMPS_NS {

class DumpCustomB200 : public DumpCustom {
 public:
  DumpCustomB200(class LAMMPS *, int, char **);
  virtual ~DumpCustomB200();
  /* B200_FIELD_* groups the columns, thresholds and region read */
  int fields_needed();

 protected:
  int count();
  class B200Link *link;
};

}

#endif
#endif
