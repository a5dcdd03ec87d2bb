/* -*- c++ -*- ----------------------------------------------------------
   pair_style lj/cut/b200 cutoff [precision fp64|mixed]

   PairLJCut (src/pair_lj_cut.h) with Pair::compute on a B200: same
   pair_coeff, pair_modify shift/mix, restart and single(); forces, energy and
   virial come from libb200md's full-list kernels (FP64 by default, or FP32
   pair math with FP64 sums with `precision mixed`).
------------------------------------------------------------------------- */

#ifdef PAIR_CLASS

PairStyle(lj/cut/b200,PairLJCutB200)

#else

#ifndef LMP_PAIR_LJ_CUT_B200_H
#define LMP_PAIR_LJ_CUT_B200_H

#include "b200_link.h"
#include "pair_lj_cut.h"

namespace LAMMPS_NS {

class PairLJCutB200 : public PairLJCut, public B200PairTables {
 public:
  PairLJCutB200(class LAMMPS *);
  ~PairLJCutB200();
  void compute(int, int);
  void settings(int, char **);
  void init_style();
  double init_one(int, int);
  int b200_upload_tables(b200_ctx *);
  int b200_precision() const { return precision; }

 private:
  int precision;
  class B200Link *link;
};

}

#endif
#endif
