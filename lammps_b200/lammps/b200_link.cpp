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
  img_applied = NULL;
  gbuf = NULL;
  nbuf = 0;
  stale = 0;
}

B200Link::~B200Link() {
  if (ctx) b200_destroy(ctx);
  memory->destroy(fbuf);
  memory->destroy(ibuf);
  memory->destroy(img_applied);
  memory->destroy(gbuf);
}

void B200Link::grow(int n) {
  if (n <= nbuf) return;
  const int old = nbuf;
  nbuf = n + n / 4 + 16;
  memory->destroy(fbuf);
  memory->destroy(ibuf);
  memory->destroy(gbuf);
  memory->create(fbuf, 3 * nbuf, "b200:fbuf");
  memory->create(ibuf, 3 * nbuf, "b200:ibuf");
  memory->create(gbuf, 12 * nbuf, "b200:gbuf");
  memory->grow(img_applied, 3 * nbuf, "b200:img_applied");
  for (int k = 3 * old; k < 3 * nbuf; k++) img_applied[k] = 0;
}

void B200Link::reset_images() {
  grow(atom->nlocal);
  for (int k = 0; k < 3 * nbuf; k++) img_applied[k] = 0;
  stale = 0;
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
  }
  apply_images(ibuf);
  stale = 0;
  long long total = 0;
  int ncalls = 0, ndanger = 0, maxneigh = 0, cap = 0;
  check(b200_neigh_stats(ctx, &total, &ncalls, &ndanger, &maxneigh, &cap), "neigh_stats");
  if (maxneigh > neighbor->oneatom) check(B200_ERR_NEIGH_OVERFLOW, "run");
}

/* The device counts each atom's box crossings since the upload; add to the
   packed image flags (src/domain.cpp:478-560 convention) the crossings not
   yet added by an earlier download of the same run.  img[3i..3i+2] are the
   device's counts of atom i. */
void B200Link::apply_images(const int *img) {
  const int n = atom->nlocal;
  for (int i = 0; i < n; i++) {
    int d[3];
    for (int k = 0; k < 3; k++) {
      d[k] = img[3 * i + k] - img_applied[3 * i + k];
      img_applied[3 * i + k] = img[3 * i + k];
    }
    imageint im = atom->image[i];
    imageint ix = (im & IMGMASK) - IMGMAX + d[0];
    imageint iy = (im >> IMGBITS & IMGMASK) - IMGMAX + d[1];
    imageint iz = (im >> IMG2BITS) - IMGMAX + d[2];
    atom->image[i] = ((imageint)(iz + IMGMAX) << IMG2BITS) |
                     ((imageint)(iy + IMGMAX) << IMGBITS) | (imageint)(ix + IMGMAX);
  }
}

void B200Link::refresh(int fields) {
  const int need = fields & stale;
  if (!need || !ctx) return;
  const int n = atom->nlocal;
  grow(n);
  int ncol = 0;
  for (int b = 1; b <= B200_FIELD_IMAGE; b <<= 1)
    if (need & b) ncol += 3;
  if (n > 0) check(b200_gather(ctx, need, n, NULL, gbuf), "gather");
  int c = 0;
  double **arr[3] = {atom->x, atom->v, atom->f};
  const int bit[3] = {B200_FIELD_X, B200_FIELD_V, B200_FIELD_F};
  for (int g = 0; g < 3; g++) {
    if (!(need & bit[g])) continue;
    double **a = arr[g];
    for (int i = 0; i < n; i++) {
      a[i][0] = gbuf[(size_t)ncol * i + c];
      a[i][1] = gbuf[(size_t)ncol * i + c + 1];
      a[i][2] = gbuf[(size_t)ncol * i + c + 2];
    }
    c += 3;
  }
  if (need & B200_FIELD_IMAGE) {
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) ibuf[3 * i + k] = (int)gbuf[(size_t)ncol * i + c + k];
    apply_images(ibuf);
  }
  stale &= ~need;
}
