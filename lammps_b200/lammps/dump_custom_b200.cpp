/* ----------------------------------------------------------------------
   dump custom/b200 -- DumpCustom fed from the device's per-atom columns.
------------------------------------------------------------------------- */

#include "dump_custom_b200.h"

#include "b200_link.h"
#include "b200md.h"

using namespace LAMMPS_NS;

DumpCustomB200::DumpCustomB200(LAMMPS *lmp, int narg, char **arg) : DumpCustom(lmp, narg, arg) {
  link = B200Link::instance(lmp);
}

DumpCustomB200::~DumpCustomB200() { B200Link::release(lmp); }

int DumpCustomB200::fields_needed() {
  const int all = B200_FIELD_X | B200_FIELD_V | B200_FIELD_F | B200_FIELD_IMAGE;
  // a threshold may test any per-atom quantity (src/dump_custom.cpp:1500-1640)
  if (nthresh > 0) return all;
  int need = iregion >= 0 ? B200_FIELD_X : 0;
  for (int i = 0; i < nfield; i++) {
    const FnPtrPack p = pack_choice[i];
    if (p == &DumpCustomB200::pack_x || p == &DumpCustomB200::pack_y ||
        p == &DumpCustomB200::pack_z || p == &DumpCustomB200::pack_xs ||
        p == &DumpCustomB200::pack_ys || p == &DumpCustomB200::pack_zs ||
        p == &DumpCustomB200::pack_xs_triclinic || p == &DumpCustomB200::pack_ys_triclinic ||
        p == &DumpCustomB200::pack_zs_triclinic)
      need |= B200_FIELD_X;
    else if (p == &DumpCustomB200::pack_xu || p == &DumpCustomB200::pack_yu ||
             p == &DumpCustomB200::pack_zu || p == &DumpCustomB200::pack_xu_triclinic ||
             p == &DumpCustomB200::pack_yu_triclinic || p == &DumpCustomB200::pack_zu_triclinic ||
             p == &DumpCustomB200::pack_xsu || p == &DumpCustomB200::pack_ysu ||
             p == &DumpCustomB200::pack_zsu || p == &DumpCustomB200::pack_xsu_triclinic ||
             p == &DumpCustomB200::pack_ysu_triclinic || p == &DumpCustomB200::pack_zsu_triclinic)
      need |= B200_FIELD_X | B200_FIELD_IMAGE;
    else if (p == &DumpCustomB200::pack_ix || p == &DumpCustomB200::pack_iy ||
             p == &DumpCustomB200::pack_iz)
      need |= B200_FIELD_IMAGE;
    else if (p == &DumpCustomB200::pack_vx || p == &DumpCustomB200::pack_vy ||
             p == &DumpCustomB200::pack_vz)
      need |= B200_FIELD_V;
    else if (p == &DumpCustomB200::pack_fx || p == &DumpCustomB200::pack_fy ||
             p == &DumpCustomB200::pack_fz)
      need |= B200_FIELD_F;
    else if (p == &DumpCustomB200::pack_compute || p == &DumpCustomB200::pack_fix ||
             p == &DumpCustomB200::pack_variable)
      return all;  // computes, fixes and variables may read any of them
    // id, type, mass, proc, molecule, custom properties: host data
  }
  return need;
}

/* DumpCustom::count (src/dump_custom.cpp:381) selects the atoms from the
   host arrays and pack() then reads them: refresh what they read first */
int DumpCustomB200::count() {
  link->refresh(fields_needed());
  return DumpCustom::count();
}
