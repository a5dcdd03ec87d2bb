/* -*- c++ -*- ----------------------------------------------------------
   pair_style eam/b200, eam/alloy/b200, eam/fs/b200 [precision fp64|mixed]

   PairEAM / PairEAMAlloy / PairEAMFS (src/MANYBODY/pair_eam*.h) with
   Pair::compute on a B200.  The potential files are read and splined by the
   reference classes (read_file, file2array, array2spline); the spline tables
   and type maps are then handed to libb200md, which runs the density,
   embedding and force passes over its own full neighbor list.  Ghost
   densities and the forward/reverse communication of rho and fp are not
   needed: each atom's density and force come from its full list.
------------------------------------------------------------------------- */

#ifdef PAIR_CLASS

PairStyle(eam/b200,PairEAMB200)
PairStyle(eam/alloy/b200,PairEAMAlloyB200)
PairStyle(eam/fs/b200,PairEAMFSB200)

#else

#ifndef LMP_PAIR_EAM_B200_H
#define LMP_PAIR_EAM_B200_H

#include "b200_link.h"
#include "pair_eam.h"
#include "pair_eam_alloy.h"
#include "pair_eam_fs.h"

namespace LAMMPS_NS {

// virtual public PairEAM: the alloy and fs forms below combine this class
// with PairEAMAlloy / PairEAMFS, which share the same PairEAM base
class PairEAMB200 : virtual public PairEAM, public B200PairTables {
 public:
  PairEAMB200(class LAMMPS *);
  virtual ~PairEAMB200();
  void compute(int, int);
  void settings(int, char **);
  void init_style();
  double init_one(int, int);
  int b200_upload_tables(b200_ctx *);
  int b200_precision() const { return precision; }
  // the style name and class for the init banner
  virtual const char *b200_style() const { return "eam/b200"; }
  virtual const char *b200_class() const { return "PairEAMB200"; }

 protected:
  int precision;
  class B200Link *link;
};

class PairEAMAlloyB200 : public PairEAMB200, public PairEAMAlloy {
 public:
  PairEAMAlloyB200(class LAMMPS *);
  virtual ~PairEAMAlloyB200() {}
  const char *b200_style() const { return "eam/alloy/b200"; }
  const char *b200_class() const { return "PairEAMAlloyB200"; }
};

class PairEAMFSB200 : public PairEAMB200, public PairEAMFS {
 public:
  PairEAMFSB200(class LAMMPS *);
  virtual ~PairEAMFSB200() {}
  const char *b200_style() const { return "eam/fs/b200"; }
  const char *b200_class() const { return "PairEAMFSB200"; }
};

}

#endif
#endif
