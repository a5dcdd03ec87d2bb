/* ----------------------------------------------------------------------
   B200 package for LAMMPS: host side of the link to libb200md.
------------------------------------------------------------------------- */

#include <cstdlib>
#include <cstring>
#include <map>

#include "b200_link.h"
#include "b200md.h"

#include "atom.h"
#include "comm.h"
#include "domain.h"
#include "error.h"
#include "force.h"
#include "lammps.h"
#include "memory.h"
#include "neighbor.h"
#include "pair.h"

using namespace LAMMPS_NS;

namespace {
std::map<LAMMPS *, B200Link *> &links() {
  static std::map<LAMMPS *, B200Link *> m;
  return m;
}
}  // namespace

B200Link *B200Link::instance(LAMMPS *lmp) {
  B200Link *&l = links()[lmp];
  if (!l) l = new B200Link(lmp);
  l->refs++;
  return l;
}

void B200Link::release(LAMMPS *lmp) {
  std::map<LAMMPS *, B200Link *>::iterator it = links().find(lmp);
  if (it == links().end()) return;
  if (--it->second->refs > 0) return;
  delete it->second;
  links().erase(it);
}

B200Link::B200Link(LAMMPS *lmp) : Pointers(lmp) {
  ctx = NULL;
  ctx_precision = -1;
  tables_dirty = 1;
  refs = 0;
  built = 0;
  nbuilt = -1;
  fbuf = NULL;
  ibuf = NULL;
  nbuf = 0;
}

B200Link::~B200Link() {
  if (ctx) b200_destroy(ctx);
  memory->destroy(fbuf);
  memory->destroy(ibuf);
}

void B200Link::grow(int n) {
  if (n <= nbuf) return;
  nbuf = n + n / 4 + 16;
  memory->destroy(fbuf);
  memory->destroy(ibuf);
  memory->create(fbuf, 3 * nbuf, "b200:fbuf");
  memory->create(ibuf, 3 * nbuf, "b200:ibuf");
}

void B200Link::check_supported(const char *style) {
  char msg[256];
  if (comm->nprocs != 1) {
    snprintf(msg, sizeof(msg), "%s runs on one MPI rank (one GPU per LAMMPS instance)", style);
    error->all(FLERR, msg);
  }
  if (domain->triclinic) {
    snprintf(msg, sizeof(msg), "%s requires an orthogonal box", style);
    error->all(FLERR, msg);
  }
  if (!domain->xperiodic || !domain->yperiodic || !domain->zperiodic) {
    snprintf(msg, sizeof(msg), "%s requires a fully periodic box", style);
    error->all(FLERR, msg);
  }
  if (atom->ntypes > 8) {
    snprintf(msg, sizeof(msg), "%s supports at most 8 atom types", style);
    error->all(FLERR, msg);
  }
}

b200_ctx *B200Link::context(int precision) {
  if (ctx && ctx_precision == precision) return ctx;
  if (ctx) b200_destroy(ctx);
  ctx = NULL;
  const char *dev = getenv("B200_DEVICE");
  int rc = b200_create(dev ? atoi(dev) : 0, precision, &ctx);
  if (rc != B200_OK) {
    char msg[512];
    snprintf(msg, sizeof(msg), "B200 context creation failed: %s", b200_last_error(ctx));
    error->all(FLERR, msg);
  }
  ctx_precision = precision;
  tables_dirty = 1;
  built = 0;
  char msg[128];
  snprintf(msg, sizeof(msg), "B200: libb200md context on CUDA device %d, %s precision",
           dev ? atoi(dev) : 0, precision == B200_PREC_MIXED ? "mixed" : "fp64");
  banner(msg);
  return ctx;
}

void B200Link::banner(const char *text) {
  if (comm->me != 0) return;
  if (screen) fprintf(screen, "%s\n", text);
  if (logfile) fprintf(logfile, "%s\n", text);
}

void B200Link::check(int status, const char *where) {
  if (status == B200_OK) return;
  char msg[640];
  if (status == B200_ERR_NEIGH_OVERFLOW)
    snprintf(msg, sizeof(msg), "Neighbor list overflow, boost neigh_modify one (%s)", where);
  else if (status == B200_ERR_LOST_ATOMS)
    snprintf(msg, sizeof(msg), "Lost atoms (%s): %s", where, b200_last_error(ctx));
  else
    snprintf(msg, sizeof(msg), "B200 %s failed (%d): %s", where, status, b200_last_error(ctx));
  error->all(FLERR, msg);
}

void B200Link::sync_settings(B200PairTables *tables) {
  context(tables->b200_precision());
  check(b200_set_box(ctx, domain->boxlo, domain->boxhi), "set_box");
  // the device list grows on demand; `neigh_modify one` is enforced on the
  // longest list after each build (pair_compute / download_state)
  check(b200_set_neighbor(ctx, neighbor->skin, neighbor->every, neighbor->delay,
                          neighbor->dist_check, 0),
        "set_neighbor");
  if (tables_dirty) {
    check(tables->b200_upload_tables(ctx), "tables");
    if (atom->mass) {
      for (int t = 1; t <= atom->ntypes; t++)
        if (atom->mass_setflag && !atom->mass_setflag[t])
          error->all(FLERR, "All masses must be set for B200 styles");
      check(b200_set_mass(ctx, atom->ntypes, atom->mass), "set_mass");
    }
    tables_dirty = 0;
  }
}

void B200Link::upload_atoms(int with_velocities) {
  const int n = atom->nlocal;
  grow(n);
  for (int i = 0; i < n; i++) ibuf[i] = (int)atom->tag[i];
  const double *x = n ? &atom->x[0][0] : NULL;
  const double *v = (with_velocities && n) ? &atom->v[0][0] : NULL;
  check(b200_upload_atoms(ctx, n, x, v, atom->type, ibuf), "upload_atoms");
}

void B200Link::pair_compute(Pair *pair, B200PairTables *tables, int eflag, int vflag) {
  const int n = atom->nlocal;
  // LAMMPS reorders and wraps atoms only when it reneighbors (pbc, exchange,
  // Atom::sort, borders in Verlet::run, src/verlet.cpp:250-270); between
  // those steps the atom set and order are fixed and the list stays valid
  const int rebuild = !ctx || ctx_precision != tables->b200_precision() || tables_dirty ||
                      !built || neighbor->ago == 0 || n != nbuilt;
  if (rebuild) {
    sync_settings(tables);
    upload_atoms(0);
    check(b200_neigh_build(ctx), "neigh_build");
    built = 1;
    nbuilt = n;
    long long total = 0;
    int ncalls = 0, ndanger = 0, maxneigh = 0, cap = 0;
    check(b200_neigh_stats(ctx, &total, &ncalls, &ndanger, &maxneigh, &cap), "neigh_stats");
    if (maxneigh > neighbor->oneatom) check(B200_ERR_NEIGH_OVERFLOW, "neigh_build");
  } else if (n > 0) {
    check(b200_update_positions(ctx, &atom->x[0][0]), "update_positions");
  }

  double eng = 0.0, vir[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double *eatom = (pair->eflag_atom && pair->eatom) ? pair->eatom : NULL;
  double *vatom = (pair->vflag_atom && pair->vatom) ? &pair->vatom[0][0] : NULL;
  check(b200_pair_compute(ctx, eflag, vflag, pair->eflag_global ? &eng : NULL,
                          pair->vflag_global ? vir : NULL, eatom, vatom),
        "pair_compute");
  grow(n);
  check(b200_download_atoms(ctx, NULL, NULL, fbuf, NULL), "download forces");
  double **f = atom->f;
  for (int i = 0; i < n; i++) {
    f[i][0] += fbuf[3 * i];
    f[i][1] += fbuf[3 * i + 1];
    f[i][2] += fbuf[3 * i + 2];
  }
  if (pair->eflag_global) pair->eng_vdwl += eng;
  if (pair->vflag_global)
    for (int k = 0; k < 6; k++) pair->virial[k] += vir[k];
}

void B200Link::download_state() {
  const int n = atom->nlocal;
  grow(n);
  double *x = n ? &atom->x[0][0] : NULL;
  double *v = n ? &atom->v[0][0] : NULL;
  check(b200_download_atoms(ctx, x, v, fbuf, ibuf), "download state");
  double **f = atom->f;
  for (int i = 0; i < n; i++) {
    f[i][0] = fbuf[3 * i];
    f[i][1] = fbuf[3 * i + 1];
    f[i][2] = fbuf[3 * i + 2];
    // the device counts box crossings since the upload; add them to the
    // packed image flags (src/domain.cpp:478-560 convention)
    imageint img = atom->image[i];
    imageint ix = (img & IMGMASK) - IMGMAX + ibuf[3 * i];
    imageint iy = (img >> IMGBITS & IMGMASK) - IMGMAX + ibuf[3 * i + 1];
    imageint iz = (img >> IMG2BITS) - IMGMAX + ibuf[3 * i + 2];
    atom->image[i] = ((imageint)(iz + IMGMAX) << IMG2BITS) |
                     ((imageint)(iy + IMGMAX) << IMGBITS) | (imageint)(ix + IMGMAX);
  }
  long long total = 0;
  int ncalls = 0, ndanger = 0, maxneigh = 0, cap = 0;
  check(b200_neigh_stats(ctx, &total, &ncalls, &ndanger, &maxneigh, &cap), "neigh_stats");
  if (maxneigh > neighbor->oneatom) check(B200_ERR_NEIGH_OVERFLOW, "run");
}
