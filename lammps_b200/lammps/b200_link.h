/* -*- c++ -*- ----------------------------------------------------------
   B200 package for LAMMPS: the link between LAMMPS's host arrays and one
   libb200md context (include/b200md.h).

   Every /b200 style of a LAMMPS instance shares one B200Link, which owns the
   device context (atoms, cell-sorted neighbor list and potential tables on
   the GPU).  Two ways of driving it:

   - per call (any run style): Pair::compute evaluates forces/energy/virial
     on the device and copies the forces back into atom->f -- the contract
     of Pair::compute(eflag,vflag) in src/pair.h:135 with the GPU package's
     device-neighbor mode as the model (src/GPU/pair_lj_cut_gpu.cpp:97-140).
     It follows LAMMPS's own reneighbor schedule: on a step where Neighbor
     has just rebuilt (neighbor->ago == 0, after pbc, exchange, sort and
     borders) it uploads the owned atoms and builds the device list;
     on the other steps it only refreshes their positions;
   - resident (run_style verlet/b200 with fix nve/b200): the whole run
     advances on the device through b200_run and host arrays are refreshed
     only on output steps.

   Limits checked at init: one MPI rank, orthogonal fully periodic box, at
   most 8 atom types, per-type masses (no rmass).
------------------------------------------------------------------------- */

#ifndef LMP_B200_LINK_H
#define LMP_B200_LINK_H

#include "pointers.h"

struct b200_ctx;

namespace LAMMPS_NS {

/* A pair style that can hand its coefficient tables to the device. */
class B200PairTables {
 public:
  virtual ~B200PairTables() {}
  /* upload the style's tables (after Pair::init) into ctx; returns a
     B200_* status */
  virtual int b200_upload_tables(b200_ctx *ctx) = 0;
  /* B200_PREC_FP64 or B200_PREC_MIXED, from the pair_style keyword */
  virtual int b200_precision() const = 0;
};

class B200Link : protected Pointers {
 public:
  /* the link of this LAMMPS instance, created on first use; every
     instance() is paired with one release(), the last one frees it */
  static B200Link *instance(class LAMMPS *);
  static void release(class LAMMPS *);

  B200Link(class LAMMPS *);
  ~B200Link();

  /* check the run can use the device at all (error->all otherwise) */
  void check_supported(const char *style);
  /* context with the requested precision on the device chosen by the
     B200_DEVICE environment variable (default 0) */
  b200_ctx *context(int precision);
  /* map a B200_* status to error->all with the library's message */
  void check(int status, const char *where);

  /* box, neighbor settings and tables, then owned atoms */
  void sync_settings(B200PairTables *tables);
  void upload_atoms(int with_velocities);
  /* per-call Pair::compute: (re)build on reneighbor steps, else refresh
     positions; then forces, energy and virial */
  void pair_compute(class Pair *pair, B200PairTables *tables, int eflag, int vflag);
  /* one line on screen and in the log file (proc 0), as the GPU package
     reports its acceleration at init */
  void banner(const char *text);

  /* resident mode: host x, v, f and image flags from the device */
  void download_state();
  /* resident mode: bring the host arrays of the B200_FIELD_* groups in
     `fields` that are behind the device (stale) up to date -- only those
     columns cross PCIe, gathered on the device (b200_gather) */
  void refresh(int fields);
  /* groups of host arrays behind the device after a partial download */
  int stale;
  /* atoms uploaded for a resident run: restart the image-flag bookkeeping */
  void reset_images();

  b200_ctx *ctx;
  int ctx_precision;
  int tables_dirty;   // tables must be re-uploaded before the next compute
  int refs;           // styles holding this link
  int built;          // the device list belongs to the current atom set
  int nbuilt;         // nlocal of that atom set

 private:
  double *fbuf;       // nlocal*3 forces in caller order
  int *ibuf;          // tags as int, image triplets
  int *img_applied;   // per atom, the device's box crossings already added to atom->image
  double *gbuf;       // gathered columns, nlocal x up to 12
  int nbuf;
  void grow(int n);
  void apply_images(const int *img);
};

}

#endif
