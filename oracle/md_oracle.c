/*
 * md_oracle.c -- CPU oracle for the short-range MD step (TEST INFRASTRUCTURE).
 *
 * Restates, in plain C, the reference's serial CPU algorithm (LAMMPS
 * "8 Aug 2014") for one periodic orthogonal box on one process.  Every
 * function cites the reference file:line it follows.  Only the tests, the
 * smoke check and bench.py's CPU-baseline leg load this code; the CUDA
 * engine never calls it.
 *
 * Floating point: build with -ffp-contract=off so that a*b+c is rounded
 * twice, as the reference's x86-64 build (no FMA) does; the neighbor
 * criterion rsq <= cutneighsq is then bit-identical to the reference.
 *
 * Threads: with nthreads > 1 the pair and neighbor loops run under OpenMP
 * with per-thread force/density copies reduced afterwards, the scheme of the
 * reference's USER-OMP package (src/USER-OMP/thr_omp.cpp:149-214).  With
 * nthreads == 1 the summation order is the serial reference order.
 */
#include "md_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXT 8
#define NSWAP 6
#define BIG 1.0e20      /* src/comm_brick.cpp:48, src/neighbor.cpp:50 */
#define SMALL 1.0e-6    /* src/neighbor.cpp:49 */
#define MAXLINE 1024
#define PS_NONE 0
#define PS_LJ 1
#define PS_EAM 2

#define MIN(a, b) ((a) < (b) ? (a) : (b))
#define MAX(a, b) ((a) > (b) ? (a) : (b))

typedef struct {
  int n, cap;
  int *list;
} ilist_t;

struct orc_sim {
  char err[256];
  int nthreads;
  /* units (src/update.cpp:118-166) */
  double boltz, mvv2e, ftm2v, nktv2p;
  int normflag;
  double dt;
  /* box */
  double boxlo[3], boxhi[3], prd[3];
  int box_set;
  /* atoms: locals [0,nlocal), ghosts [nlocal,nlocal+nghost) */
  int nlocal, nghost, nmax;
  double *x, *v, *f;
  int *type, *tag, *image;  /* image: 3 ints per atom */
  int *gowner, *gimg;       /* per ghost: owner local index and image */
  int ntypes;
  double mass[MAXT + 1];
  /* swaps of CommBrick for one process (src/comm_brick.cpp:151-398) */
  int nswap;
  ilist_t sendlist[NSWAP];
  int firstrecv[NSWAP], recvnum[NSWAP], pbc[NSWAP][3];
  double slablo[NSWAP], slabhi[NSWAP];
  /* pair style */
  int pstyle;
  double cut_global;
  int offset_flag;
  double eps[MAXT + 1][MAXT + 1], sig[MAXT + 1][MAXT + 1], cut[MAXT + 1][MAXT + 1];
  int setflag[MAXT + 1][MAXT + 1];
  double cutsq[MAXT + 1][MAXT + 1];
  double lj1[MAXT + 1][MAXT + 1], lj2[MAXT + 1][MAXT + 1], lj3[MAXT + 1][MAXT + 1],
      lj4[MAXT + 1][MAXT + 1], offset[MAXT + 1][MAXT + 1];
  /* eam */
  int eam_kind; /* 0 funcfl, 1 setfl, 2 fs */
  int nfuncfl;
  struct {
    int nrho, nr;
    double drho, dr, cut, mass;
    double *frho, *rhor, *zr;
  } ffl[MAXT];
  int map[MAXT + 1];
  int nelements;
  double *sf_frho, *sf_rhor, *sf_z2r, *sf_mass; /* setfl/fs raw arrays */
  int sf_nrho, sf_nr;
  double sf_drho, sf_dr, sf_cut;
  int nrho, nr, nfrho, nrhor, nz2r;
  double drho, dr, rdr, rdrho, rhomax, cutmax, cutforcesq;
  double *frho, *rhor, *z2r;
  double *frho_spline, *rhor_spline, *z2r_spline;
  int type2frho[MAXT + 1], type2rhor[MAXT + 1][MAXT + 1], type2z2r[MAXT + 1][MAXT + 1];
  double *rho, *fp;
  /* neighbor */
  double skin, cutneighmax, cutneighmaxsq, triggersq;
  double cutneighsq[MAXT + 1][MAXT + 1];
  int every, delay, dist_check, ago, ncalls, ndanger;
  int nbinx, nbiny, nbinz, mbinx, mbiny, mbinz, mbinxlo, mbinylo, mbinzlo, mbins;
  double binsizex, binsizey, binsizez, bininvx, bininvy, bininvz;
  int *binhead, *bins;
  int *stencil, nstencil;
  int *numneigh;
  int **firstneigh;
  int nbuf;
  ilist_t *neighbuf; /* one growable page per thread */
  double *xhold;
  /* atom sort (src/atom.cpp:1575-1742) */
  int sortfreq;
  long long nextsort;
  /* energy / virial */
  double eng_vdwl, virial[6];
  double *eatom, *vatom;
  int evflag, eflag_global, eflag_atom, vflag_global, vflag_atom, vflag_fdotr;
  /* time */
  long long ntimestep, laststep;
  int thermo_every;
  double *rows;
  int nrows, maxrows;
  double temp_scalar, press_scalar;
  int setup_done;
};

/* ------------------------------------------------------------------ */

static int fail(orc_sim *s, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(s->err, sizeof(s->err), fmt, ap);
  va_end(ap);
  return -1;
}

static void *xrealloc(void *p, size_t n) {
  void *q = realloc(p, n ? n : 1);
  if (!q) {
    fprintf(stderr, "md_oracle: out of memory\n");
    abort();
  }
  return q;
}

static void il_push(ilist_t *l, int v) {
  if (l->n == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 1024;
    l->list = (int *)xrealloc(l->list, sizeof(int) * (size_t)l->cap);
  }
  l->list[l->n++] = v;
}

static void grow_atoms(orc_sim *s, int n) {
  if (n <= s->nmax) return;
  int nm = s->nmax ? s->nmax : 1024;
  while (nm < n) nm *= 2;
  s->x = (double *)xrealloc(s->x, sizeof(double) * 3 * (size_t)nm);
  s->v = (double *)xrealloc(s->v, sizeof(double) * 3 * (size_t)nm);
  s->f = (double *)xrealloc(s->f, sizeof(double) * 3 * (size_t)nm);
  s->type = (int *)xrealloc(s->type, sizeof(int) * (size_t)nm);
  s->tag = (int *)xrealloc(s->tag, sizeof(int) * (size_t)nm);
  s->image = (int *)xrealloc(s->image, sizeof(int) * 3 * (size_t)nm);
  s->gowner = (int *)xrealloc(s->gowner, sizeof(int) * (size_t)nm);
  s->gimg = (int *)xrealloc(s->gimg, sizeof(int) * 3 * (size_t)nm);
  s->rho = (double *)xrealloc(s->rho, sizeof(double) * (size_t)nm);
  s->fp = (double *)xrealloc(s->fp, sizeof(double) * (size_t)nm);
  s->eatom = (double *)xrealloc(s->eatom, sizeof(double) * (size_t)nm);
  s->vatom = (double *)xrealloc(s->vatom, sizeof(double) * 6 * (size_t)nm);
  s->bins = (int *)xrealloc(s->bins, sizeof(int) * (size_t)nm);
  s->nmax = nm;
}

/* ------------------------------------------------------------------ */
/* creation and settings                                               */

orc_sim *orc_create(int unit_style) {
  orc_sim *s = (orc_sim *)calloc(1, sizeof(orc_sim));
  s->nthreads = 1;
  if (unit_style == 1) { /* metal: src/update.cpp:160-175 */
    s->boltz = 8.617343e-5;
    s->mvv2e = 1.0364269e-4;
    s->ftm2v = 1.0 / 1.0364269e-4;
    s->nktv2p = 1.6021765e6;
    s->dt = 0.001;
    s->skin = 2.0;
    s->normflag = 0;
  } else { /* lj: src/update.cpp:118-137 */
    s->boltz = 1.0;
    s->mvv2e = 1.0;
    s->ftm2v = 1.0;
    s->nktv2p = 1.0;
    s->dt = 0.005;
    s->skin = 0.3;
    s->normflag = 1; /* src/thermo.cpp:191 */
  }
  /* neighbor defaults: src/neighbor.cpp:78-82; atom sort src/atom.cpp:63 */
  s->every = 1;
  s->delay = 10;
  s->dist_check = 1;
  s->sortfreq = 1000;
  for (int i = 0; i <= MAXT; i++) s->map[i] = -1;
  return s;
}

static void free_eam(orc_sim *s) {
  for (int i = 0; i < s->nfuncfl; i++) {
    free(s->ffl[i].frho);
    free(s->ffl[i].rhor);
    free(s->ffl[i].zr);
  }
  s->nfuncfl = 0;
  free(s->sf_frho); free(s->sf_rhor); free(s->sf_z2r); free(s->sf_mass);
  s->sf_frho = s->sf_rhor = s->sf_z2r = s->sf_mass = NULL;
  free(s->frho); free(s->rhor); free(s->z2r);
  free(s->frho_spline); free(s->rhor_spline); free(s->z2r_spline);
  s->frho = s->rhor = s->z2r = NULL;
  s->frho_spline = s->rhor_spline = s->z2r_spline = NULL;
}

void orc_destroy(orc_sim *s) {
  if (!s) return;
  free(s->x); free(s->v); free(s->f); free(s->type); free(s->tag); free(s->image);
  free(s->gowner); free(s->gimg); free(s->rho); free(s->fp); free(s->eatom); free(s->vatom);
  free(s->bins); free(s->binhead); free(s->stencil); free(s->numneigh); free(s->firstneigh);
  for (int t = 0; t < s->nbuf; t++) free(s->neighbuf[t].list);
  free(s->neighbuf);
  free(s->xhold);
  for (int i = 0; i < NSWAP; i++) free(s->sendlist[i].list);
  free(s->rows);
  free_eam(s);
  free(s);
}

const char *orc_error(orc_sim *s) { return s->err; }
void orc_set_threads(orc_sim *s, int n) { s->nthreads = n > 0 ? n : 1; }
void orc_set_timestep(orc_sim *s, double dt) { s->dt = dt; }
void orc_set_thermo(orc_sim *s, int every) { s->thermo_every = every; }
void orc_set_mass(orc_sim *s, int itype, double m) {
  if (itype >= 1 && itype <= MAXT) s->mass[itype] = m;
}
void orc_set_neighbor(orc_sim *s, double skin, int every, int delay, int check, int sortfreq) {
  s->skin = skin;
  s->every = every;
  s->delay = delay;
  s->dist_check = check;
  s->sortfreq = sortfreq;
}

/* Domain::set_global_box: prd = hi - lo (src/domain.cpp:213-217) */
int orc_set_box(orc_sim *s, const double lo[3], const double hi[3]) {
  for (int d = 0; d < 3; d++) {
    s->boxlo[d] = lo[d];
    s->boxhi[d] = hi[d];
    s->prd[d] = hi[d] - lo[d];
    if (!(s->prd[d] > 0.0)) return fail(s, "invalid box");
  }
  s->box_set = 1;
  return 0;
}

int orc_set_atoms(orc_sim *s, int n, int ntypes, const double *x, const double *v,
                  const int *type, const int *tag) {
  if (n < 0 || ntypes < 1 || ntypes > MAXT) return fail(s, "bad atom count or ntypes");
  grow_atoms(s, n + 16);
  s->nlocal = n;
  s->nghost = 0;
  s->ntypes = ntypes;
  memcpy(s->x, x, sizeof(double) * 3 * (size_t)n);
  if (v) memcpy(s->v, v, sizeof(double) * 3 * (size_t)n);
  else memset(s->v, 0, sizeof(double) * 3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    s->type[i] = type ? type[i] : 1;
    if (s->type[i] < 1 || s->type[i] > ntypes) return fail(s, "atom type out of range");
    s->tag[i] = tag ? tag[i] : i + 1;
    s->image[3 * i] = s->image[3 * i + 1] = s->image[3 * i + 2] = 0;
  }
  memset(s->f, 0, sizeof(double) * 3 * (size_t)n);
  s->setup_done = 0;
  return 0;
}

/* ------------------------------------------------------------------ */
/* input generators                                                    */

/* fcc basis src/lattice.cpp:84-94; loop order k,j,i,basis
   src/create_atoms.cpp:726-760; lattice2box with identity orientation
   src/lattice.cpp:468-485 */
int orc_lattice(int style, int nx, int ny, int nz, double scale, double *x) {
  static const double sc[1][3] = {{0.0, 0.0, 0.0}};
  static const double bcc[2][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.5}};
  static const double fcc[4][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5},
                                   {0.0, 0.5, 0.5}};
  const double(*basis)[3] = style == 0 ? sc : (style == 1 ? bcc : fcc);
  int nb = style == 0 ? 1 : (style == 1 ? 2 : 4);
  int n = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int m = 0; m < nb; m++) {
          double a = i + basis[m][0], b = j + basis[m][1], c = k + basis[m][2];
          /* primitive = identity, rotaterow = identity, origin = 0 */
          double x1 = 1.0 * a + 0.0 * b + 0.0 * c;
          double y1 = 0.0 * a + 1.0 * b + 0.0 * c;
          double z1 = 0.0 * a + 0.0 * b + 1.0 * c;
          x1 *= scale;
          y1 *= scale;
          z1 *= scale;
          x[3 * n] = 1.0 * x1 + 0.0 * y1 + 0.0 * z1 + 0.0;
          x[3 * n + 1] = 0.0 * x1 + 1.0 * y1 + 0.0 * z1 + 0.0;
          x[3 * n + 2] = 0.0 * x1 + 0.0 * y1 + 1.0 * z1 + 0.0;
          n++;
        }
  return n;
}

/* scale = (nbasis / (Vprimitive * rho*))^(1/3)  (src/lattice.cpp:249-256) */
double orc_lj_lattice_scale(int style, double rhostar) {
  int nb = style == 0 ? 1 : (style == 1 ? 2 : 4);
  double volume = 1.0;
  return pow(nb / volume / rhostar, 1.0 / 3.0);
}

/* RanPark: Park-Miller minimal standard (src/random_park.cpp:42-76) */
typedef struct {
  int seed, save;
  double second;
} ranpark;

static double rp_uniform(ranpark *r) {
  const int IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836;
  const double AM = 1.0 / IM;
  int k = r->seed / IQ;
  r->seed = IA * (r->seed - k * IQ) - IR * k;
  if (r->seed < 0) r->seed += IM;
  return AM * r->seed;
}

static double rp_gaussian(ranpark *r) {
  double first, v1, v2, rsq, fac;
  if (!r->save) {
    int again = 1;
    while (again) {
      v1 = 2.0 * rp_uniform(r) - 1.0;
      v2 = 2.0 * rp_uniform(r) - 1.0;
      rsq = v1 * v1 + v2 * v2;
      if (rsq < 1.0 && rsq != 0.0) again = 0;
    }
    fac = sqrt(-2.0 * log(rsq) / rsq);
    r->second = v1 * fac;
    first = v2 * fac;
    r->save = 1;
  } else {
    first = r->second;
    r->save = 0;
  }
  return first;
}

/* Jenkins one-at-a-time hash of the seed and coordinate bytes, 27-bit seed,
   5 warm-up draws (src/random_park.cpp:94-130).  Bytes are read as signed
   char, as the reference's `char *` does on x86-64. */
static void rp_reset_geom(ranpark *r, int ibase, const double *coord) {
  unsigned int hash = 0;
  const signed char *str = (const signed char *)&ibase;
  for (int i = 0; i < (int)sizeof(int); i++) {
    hash += (unsigned int)(int)str[i];
    hash += (hash << 10);
    hash ^= (hash >> 6);
  }
  str = (const signed char *)coord;
  for (int i = 0; i < 3 * (int)sizeof(double); i++) {
    hash += (unsigned int)(int)str[i];
    hash += (hash << 10);
    hash ^= (hash >> 6);
  }
  hash += (hash << 3);
  hash ^= (hash >> 11);
  hash += (hash << 15);
  r->seed = (int)(hash & 0x7ffffff);
  if (!r->seed) r->seed = 1;
  for (int i = 0; i < 5; i++) rp_uniform(r);
  r->save = 0;
}

/* ComputeTemp::compute_scalar (src/compute_temp.cpp:59-89), dof = 3N-3 */
static double temp_scalar(orc_sim *s) {
  double t = 0.0;
  for (int i = 0; i < s->nlocal; i++) {
    const double *v = s->v + 3 * i;
    t += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * s->mass[s->type[i]];
  }
  double dof = 3.0 * s->nlocal - 3.0;
  double tfactor = dof > 0.0 ? s->mvv2e / (dof * s->boltz) : 0.0;
  return t * tfactor;
}

/* Velocity::create (src/velocity.cpp:136-340) with zero_momentum
   (:688-713, Group::mass/vcm src/group.cpp:782-805,1090-1128) and
   rescale (:666-682) */
int orc_velocity_create(orc_sim *s, double t_desired, int seed, int gaussian,
                        int loop_geom, int mom) {
  if (seed <= 0) return fail(s, "Illegal velocity create command");
  int n = s->nlocal;
  ranpark r = {1, 0, 0.0};
  if (loop_geom) {
    for (int i = 0; i < n; i++) {
      rp_reset_geom(&r, seed, s->x + 3 * i);
      double vx, vy, vz;
      if (!gaussian) {
        vx = rp_uniform(&r);
        vy = rp_uniform(&r);
        vz = rp_uniform(&r);
      } else {
        vx = rp_gaussian(&r);
        vy = rp_gaussian(&r);
        vz = rp_gaussian(&r);
      }
      double factor = 1.0 / sqrt(s->mass[s->type[i]]);
      s->v[3 * i] = vx * factor;
      s->v[3 * i + 1] = vy * factor;
      s->v[3 * i + 2] = vz * factor;
    }
  } else {
    /* loop all: one RNG stream over tags 1..natoms */
    int *map = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    for (int i = 0; i <= n; i++) map[i] = -1;
    for (int i = 0; i < n; i++)
      if (s->tag[i] >= 1 && s->tag[i] <= n) map[s->tag[i]] = i;
    r.seed = seed;
    for (int t = 1; t <= n; t++) {
      double vx, vy, vz;
      if (!gaussian) {
        vx = rp_uniform(&r);
        vy = rp_uniform(&r);
        vz = rp_uniform(&r);
      } else {
        vx = rp_gaussian(&r);
        vy = rp_gaussian(&r);
        vz = rp_gaussian(&r);
      }
      int m = map[t];
      if (m >= 0) {
        double factor = 1.0 / sqrt(s->mass[s->type[m]]);
        s->v[3 * m] = vx * factor;
        s->v[3 * m + 1] = vy * factor;
        s->v[3 * m + 2] = vz * factor;
      }
    }
    free(map);
  }
  if (mom) {
    double masstotal = 0.0, p[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; i++) masstotal += s->mass[s->type[i]];
    for (int i = 0; i < n; i++) {
      double m = s->mass[s->type[i]];
      p[0] += s->v[3 * i] * m;
      p[1] += s->v[3 * i + 1] * m;
      p[2] += s->v[3 * i + 2] * m;
    }
    if (masstotal > 0.0) {
      p[0] /= masstotal;
      p[1] /= masstotal;
      p[2] /= masstotal;
    }
    for (int i = 0; i < n; i++) {
      s->v[3 * i] -= p[0];
      s->v[3 * i + 1] -= p[1];
      s->v[3 * i + 2] -= p[2];
    }
  }
  double t = temp_scalar(s);
  if (t == 0.0) return fail(s, "Attempting to rescale a 0.0 temperature");
  double factor = sqrt(t_desired / t);
  for (int i = 0; i < 3 * n; i++) s->v[i] *= factor;
  return 0;
}

/* ------------------------------------------------------------------ */
/* pair style settings                                                 */

/* pair_style lj/cut (src/pair_lj_cut.cpp:428-476) */
int orc_pair_lj_cut(orc_sim *s, double cut_global, int shift) {
  s->pstyle = PS_LJ;
  s->cut_global = cut_global;
  s->offset_flag = shift;
  memset(s->setflag, 0, sizeof(s->setflag));
  return 0;
}

int orc_pair_lj_coeff(orc_sim *s, int i, int j, double eps, double sigma, double cut) {
  if (s->pstyle != PS_LJ) return fail(s, "pair style is not lj/cut");
  if (i < 1 || j < 1 || i > MAXT || j > MAXT) return fail(s, "bad type");
  if (i > j) { int t = i; i = j; j = t; }
  s->eps[i][j] = eps;
  s->sig[i][j] = sigma;
  s->cut[i][j] = cut < 0.0 ? s->cut_global : cut;
  s->setflag[i][j] = 1;
  return 0;
}

/* PairLJCut::init_one with geometric mixing (src/pair_lj_cut.cpp:545-570,
   src/pair.cpp:639-664) and Pair::init cutsq = cut^2 (src/pair.cpp:214-224) */
static int init_lj(orc_sim *s) {
  int n = s->ntypes;
  for (int i = 1; i <= n; i++)
    if (!s->setflag[i][i]) return fail(s, "All pair coeffs are not set");
  for (int i = 1; i <= n; i++)
    for (int j = i; j <= n; j++) {
      if (!s->setflag[i][j]) {
        s->eps[i][j] = sqrt(s->eps[i][i] * s->eps[j][j]);
        s->sig[i][j] = sqrt(s->sig[i][i] * s->sig[j][j]);
        s->cut[i][j] = sqrt(s->cut[i][i] * s->cut[j][j]);
      }
      double e = s->eps[i][j], sg = s->sig[i][j], c = s->cut[i][j];
      s->lj1[i][j] = 48.0 * e * pow(sg, 12.0);
      s->lj2[i][j] = 24.0 * e * pow(sg, 6.0);
      s->lj3[i][j] = 4.0 * e * pow(sg, 12.0);
      s->lj4[i][j] = 4.0 * e * pow(sg, 6.0);
      if (s->offset_flag) {
        double ratio = sg / c;
        s->offset[i][j] = 4.0 * e * (pow(ratio, 12.0) - pow(ratio, 6.0));
      } else
        s->offset[i][j] = 0.0;
      s->lj1[j][i] = s->lj1[i][j];
      s->lj2[j][i] = s->lj2[i][j];
      s->lj3[j][i] = s->lj3[i][j];
      s->lj4[j][i] = s->lj4[i][j];
      s->offset[j][i] = s->offset[i][j];
      s->cutsq[i][j] = s->cutsq[j][i] = c * c;
    }
  return 0;
}

/* PairEAM::grab (src/MANYBODY/pair_eam.cpp:759-771) */
static int grab(FILE *fp, int n, double *list) {
  char line[MAXLINE];
  int i = 0;
  while (i < n) {
    if (!fgets(line, MAXLINE, fp)) return -1;
    char *ptr = strtok(line, " \t\n\r\f");
    if (!ptr) continue;
    list[i++] = atof(ptr);
    while ((ptr = strtok(NULL, " \t\n\r\f")) && i < n) list[i++] = atof(ptr);
  }
  return 0;
}

/* PairEAM::read_file for DYNAMO funcfl (src/MANYBODY/pair_eam.cpp:433-481) */
static int read_funcfl(orc_sim *s, const char *path, int idx) {
  FILE *fp = fopen(path, "r");
  if (!fp) return fail(s, "Cannot open EAM potential file %s", path);
  char line[MAXLINE];
  int tmp;
  if (!fgets(line, MAXLINE, fp) || !fgets(line, MAXLINE, fp)) goto bad;
  sscanf(line, "%d %lg", &tmp, &s->ffl[idx].mass);
  if (!fgets(line, MAXLINE, fp)) goto bad;
  if (sscanf(line, "%d %lg %d %lg %lg", &s->ffl[idx].nrho, &s->ffl[idx].drho, &s->ffl[idx].nr,
             &s->ffl[idx].dr, &s->ffl[idx].cut) != 5)
    goto bad;
  s->ffl[idx].frho = (double *)calloc((size_t)s->ffl[idx].nrho + 1, sizeof(double));
  s->ffl[idx].rhor = (double *)calloc((size_t)s->ffl[idx].nr + 1, sizeof(double));
  s->ffl[idx].zr = (double *)calloc((size_t)s->ffl[idx].nr + 1, sizeof(double));
  if (grab(fp, s->ffl[idx].nrho, &s->ffl[idx].frho[1])) goto bad;
  if (grab(fp, s->ffl[idx].nr, &s->ffl[idx].zr[1])) goto bad;
  if (grab(fp, s->ffl[idx].nr, &s->ffl[idx].rhor[1])) goto bad;
  fclose(fp);
  return 0;
bad:
  fclose(fp);
  return fail(s, "Bad EAM potential file %s", path);
}

int orc_pair_eam_funcfl(orc_sim *s, int nfiles, const char **files, const int *type2file) {
  free_eam(s);
  if (nfiles < 1 || nfiles > MAXT) return fail(s, "bad funcfl count");
  s->pstyle = PS_EAM;
  s->eam_kind = 0;
  for (int i = 0; i < nfiles; i++) {
    s->nfuncfl = i + 1;
    if (read_funcfl(s, files[i], i)) return -1;
  }
  for (int t = 1; t <= MAXT; t++) s->map[t] = -1;
  for (int t = 1; t <= MAXT; t++)
    if (type2file[t - 1] >= 0) {
      s->map[t] = type2file[t - 1];
      s->mass[t] = s->ffl[type2file[t - 1]].mass; /* atom->set_mass (:384) */
    }
  return 0;
}

/* PairEAMAlloy/PairEAMFS::read_file (src/MANYBODY/pair_eam_alloy.cpp:115-207,
   src/MANYBODY/pair_eam_fs.cpp) */
int orc_pair_eam_setfl(orc_sim *s, const char *path, int fs, const int *map) {
  free_eam(s);
  s->pstyle = PS_EAM;
  s->eam_kind = fs ? 2 : 1;
  FILE *fp = fopen(path, "r");
  if (!fp) return fail(s, "Cannot open EAM potential file %s", path);
  char line[MAXLINE];
  int ne;
  for (int k = 0; k < 4; k++)
    if (!fgets(line, MAXLINE, fp)) goto bad;
  if (sscanf(line, "%d", &ne) != 1 || ne < 1 || ne > MAXT) goto bad;
  s->nelements = ne;
  if (!fgets(line, MAXLINE, fp)) goto bad;
  if (sscanf(line, "%d %lg %d %lg %lg", &s->sf_nrho, &s->sf_drho, &s->sf_nr, &s->sf_dr,
             &s->sf_cut) != 5)
    goto bad;
  {
    int nrho = s->sf_nrho, nr = s->sf_nr;
    s->sf_mass = (double *)calloc((size_t)ne, sizeof(double));
    s->sf_frho = (double *)calloc((size_t)ne * (nrho + 1), sizeof(double));
    int nrhor_f = fs ? ne * ne : ne;
    s->sf_rhor = (double *)calloc((size_t)nrhor_f * (nr + 1), sizeof(double));
    s->sf_z2r = (double *)calloc((size_t)ne * ne * (nr + 1), sizeof(double));
    for (int i = 0; i < ne; i++) {
      int tmp;
      if (!fgets(line, MAXLINE, fp)) goto bad;
      sscanf(line, "%d %lg", &tmp, &s->sf_mass[i]);
      if (grab(fp, nrho, &s->sf_frho[(size_t)i * (nrho + 1) + 1])) goto bad;
      if (fs) {
        for (int j = 0; j < ne; j++)
          if (grab(fp, nr, &s->sf_rhor[((size_t)i * ne + j) * (nr + 1) + 1])) goto bad;
      } else if (grab(fp, nr, &s->sf_rhor[(size_t)i * (nr + 1) + 1]))
        goto bad;
    }
    for (int i = 0; i < ne; i++)
      for (int j = 0; j <= i; j++)
        if (grab(fp, nr, &s->sf_z2r[((size_t)i * ne + j) * (nr + 1) + 1])) goto bad;
  }
  fclose(fp);
  for (int t = 1; t <= MAXT; t++) s->map[t] = -1;
  for (int t = 1; t <= MAXT; t++)
    if (map[t - 1] >= 0) {
      if (map[t - 1] >= ne) return fail(s, "No matching element in EAM potential file");
      s->map[t] = map[t - 1];
      s->mass[t] = s->sf_mass[map[t - 1]];
    }
  return 0;
bad:
  fclose(fp);
  return fail(s, "Bad EAM potential file %s", path);
}

/* PairEAM::interpolate (src/MANYBODY/pair_eam.cpp:723-751) */
static void interpolate(int n, double delta, const double *f, double *spl) {
#define S(m, k) spl[(size_t)(m)*7 + (k)]
  for (int m = 1; m <= n; m++) S(m, 6) = f[m];
  S(1, 5) = S(2, 6) - S(1, 6);
  S(2, 5) = 0.5 * (S(3, 6) - S(1, 6));
  S(n - 1, 5) = 0.5 * (S(n, 6) - S(n - 2, 6));
  S(n, 5) = S(n, 6) - S(n - 1, 6);
  for (int m = 3; m <= n - 2; m++)
    S(m, 5) = ((S(m - 2, 6) - S(m + 2, 6)) + 8.0 * (S(m + 1, 6) - S(m - 1, 6))) / 12.0;
  for (int m = 1; m <= n - 1; m++) {
    S(m, 4) = 3.0 * (S(m + 1, 6) - S(m, 6)) - 2.0 * S(m, 5) - S(m + 1, 5);
    S(m, 3) = S(m, 5) + S(m + 1, 5) - 2.0 * (S(m + 1, 6) - S(m, 6));
  }
  S(n, 4) = 0.0;
  S(n, 3) = 0.0;
  for (int m = 1; m <= n; m++) {
    S(m, 2) = S(m, 5) / delta;
    S(m, 1) = 2.0 * S(m, 4) / delta;
    S(m, 0) = 3.0 * S(m, 3) / delta;
  }
#undef S
}

static double lagrange4(const double *tab, int ntab, double dtab, double r) {
  const double sixth = 1.0 / 6.0;
  double p = r / dtab + 1.0;
  int k = (int)p;
  k = MIN(k, ntab - 2);
  k = MAX(k, 2);
  p -= k;
  p = MIN(p, 2.0);
  double cof1 = -sixth * p * (p - 1.0) * (p - 2.0);
  double cof2 = 0.5 * (p * p - 1.0) * (p - 2.0);
  double cof3 = -0.5 * p * (p + 1.0) * (p - 2.0);
  double cof4 = sixth * p * (p * p - 1.0);
  return cof1 * tab[k - 1] + cof2 * tab[k] + cof3 * tab[k + 1] + cof4 * tab[k + 2];
}

static int type2z2r_index(int irow, int icol) {
  if (irow < icol) { int t = irow; irow = icol; icol = t; }
  int n = 0;
  for (int m = 0; m < irow; m++) n += m + 1;
  return n + icol;
}

/* PairEAM::file2array (src/MANYBODY/pair_eam.cpp:488-694),
   PairEAMAlloy::file2array (src/MANYBODY/pair_eam_alloy.cpp:213-326),
   PairEAMFS::file2array (src/MANYBODY/pair_eam_fs.cpp), then array2spline
   (src/MANYBODY/pair_eam.cpp:698-719) and init_one (:411-427) */
static int init_eam(orc_sim *s) {
  int nt = s->ntypes;
  for (int t = 1; t <= nt; t++)
    if (s->map[t] < 0) return fail(s, "All pair coeffs are not set");
  free(s->frho); free(s->rhor); free(s->z2r);
  if (s->eam_kind == 0) {
    double rmax = 0.0;
    s->dr = s->drho = s->rhomax = 0.0;
    for (int i = 0; i < s->nfuncfl; i++) {
      int active = 0;
      for (int j = 1; j <= nt; j++)
        if (s->map[j] == i) active = 1;
      if (!active) continue;
      s->dr = MAX(s->dr, s->ffl[i].dr);
      s->drho = MAX(s->drho, s->ffl[i].drho);
      rmax = MAX(rmax, (s->ffl[i].nr - 1) * s->ffl[i].dr);
      s->rhomax = MAX(s->rhomax, (s->ffl[i].nrho - 1) * s->ffl[i].drho);
    }
    s->nr = (int)(rmax / s->dr + 0.5);
    s->nrho = (int)(s->rhomax / s->drho + 0.5);
    s->nfrho = s->nfuncfl + 1;
    s->frho = (double *)calloc((size_t)s->nfrho * (s->nrho + 1), sizeof(double));
    for (int i = 0; i < s->nfuncfl; i++)
      for (int m = 1; m <= s->nrho; m++) {
        double r = (m - 1) * s->drho;
        s->frho[(size_t)i * (s->nrho + 1) + m] =
            lagrange4(s->ffl[i].frho, s->ffl[i].nrho, s->ffl[i].drho, r);
      }
    for (int t = 1; t <= nt; t++) s->type2frho[t] = s->map[t] >= 0 ? s->map[t] : s->nfrho - 1;
    s->nrhor = s->nfuncfl;
    s->rhor = (double *)calloc((size_t)s->nrhor * (s->nr + 1), sizeof(double));
    for (int i = 0; i < s->nfuncfl; i++)
      for (int m = 1; m <= s->nr; m++) {
        double r = (m - 1) * s->dr;
        s->rhor[(size_t)i * (s->nr + 1) + m] =
            lagrange4(s->ffl[i].rhor, s->ffl[i].nr, s->ffl[i].dr, r);
      }
    for (int i = 1; i <= nt; i++)
      for (int j = 1; j <= nt; j++) s->type2rhor[i][j] = s->map[i];
    s->nz2r = s->nfuncfl * (s->nfuncfl + 1) / 2;
    s->z2r = (double *)calloc((size_t)s->nz2r * (s->nr + 1), sizeof(double));
    int n = 0;
    for (int i = 0; i < s->nfuncfl; i++)
      for (int j = 0; j <= i; j++) {
        for (int m = 1; m <= s->nr; m++) {
          double r = (m - 1) * s->dr;
          double zri = lagrange4(s->ffl[i].zr, s->ffl[i].nr, s->ffl[i].dr, r);
          double zrj = lagrange4(s->ffl[j].zr, s->ffl[j].nr, s->ffl[j].dr, r);
          s->z2r[(size_t)n * (s->nr + 1) + m] = 27.2 * 0.529 * zri * zrj;
        }
        n++;
      }
    s->cutmax = 0.0;
    for (int m = 0; m < s->nfuncfl; m++) s->cutmax = MAX(s->cutmax, s->ffl[m].cut);
  } else {
    int ne = s->nelements, fs = s->eam_kind == 2;
    s->nrho = s->sf_nrho;
    s->nr = s->sf_nr;
    s->drho = s->sf_drho;
    s->dr = s->sf_dr;
    s->rhomax = (s->nrho - 1) * s->drho;
    s->nfrho = ne + 1;
    s->frho = (double *)calloc((size_t)s->nfrho * (s->nrho + 1), sizeof(double));
    for (int i = 0; i < ne; i++)
      for (int m = 1; m <= s->nrho; m++)
        s->frho[(size_t)i * (s->nrho + 1) + m] = s->sf_frho[(size_t)i * (s->nrho + 1) + m];
    for (int t = 1; t <= nt; t++) s->type2frho[t] = s->map[t] >= 0 ? s->map[t] : s->nfrho - 1;
    s->nrhor = fs ? ne * ne : ne;
    s->rhor = (double *)calloc((size_t)s->nrhor * (s->nr + 1), sizeof(double));
    for (int i = 0; i < s->nrhor; i++)
      for (int m = 1; m <= s->nr; m++)
        s->rhor[(size_t)i * (s->nr + 1) + m] = s->sf_rhor[(size_t)i * (s->nr + 1) + m];
    for (int i = 1; i <= nt; i++)
      for (int j = 1; j <= nt; j++)
        s->type2rhor[i][j] = fs ? s->map[i] * ne + s->map[j] : s->map[i];
    s->nz2r = ne * (ne + 1) / 2;
    s->z2r = (double *)calloc((size_t)s->nz2r * (s->nr + 1), sizeof(double));
    int n = 0;
    for (int i = 0; i < ne; i++)
      for (int j = 0; j <= i; j++) {
        for (int m = 1; m <= s->nr; m++)
          s->z2r[(size_t)n * (s->nr + 1) + m] = s->sf_z2r[((size_t)i * ne + j) * (s->nr + 1) + m];
        n++;
      }
    s->cutmax = s->sf_cut;
  }
  for (int i = 1; i <= nt; i++)
    for (int j = 1; j <= nt; j++)
      s->type2z2r[i][j] = type2z2r_index(s->map[i], s->map[j]);
  /* array2spline */
  s->rdr = 1.0 / s->dr;
  s->rdrho = 1.0 / s->drho;
  free(s->frho_spline); free(s->rhor_spline); free(s->z2r_spline);
  s->frho_spline = (double *)calloc((size_t)s->nfrho * (s->nrho + 1) * 7, sizeof(double));
  s->rhor_spline = (double *)calloc((size_t)s->nrhor * (s->nr + 1) * 7, sizeof(double));
  s->z2r_spline = (double *)calloc((size_t)s->nz2r * (s->nr + 1) * 7, sizeof(double));
  for (int i = 0; i < s->nfrho; i++)
    interpolate(s->nrho, s->drho, s->frho + (size_t)i * (s->nrho + 1),
                s->frho_spline + (size_t)i * (s->nrho + 1) * 7);
  for (int i = 0; i < s->nrhor; i++)
    interpolate(s->nr, s->dr, s->rhor + (size_t)i * (s->nr + 1),
                s->rhor_spline + (size_t)i * (s->nr + 1) * 7);
  for (int i = 0; i < s->nz2r; i++)
    interpolate(s->nr, s->dr, s->z2r + (size_t)i * (s->nr + 1),
                s->z2r_spline + (size_t)i * (s->nr + 1) * 7);
  s->cutforcesq = s->cutmax * s->cutmax;
  for (int i = 1; i <= nt; i++)
    for (int j = 1; j <= nt; j++) s->cutsq[i][j] = s->cutmax * s->cutmax;
  return 0;
}

int orc_eam_info(orc_sim *s, int *ints, double *dbls) {
  if (s->pstyle != PS_EAM || !s->frho_spline) return fail(s, "eam not initialised");
  ints[0] = s->nrho; ints[1] = s->nr; ints[2] = s->nfrho; ints[3] = s->nrhor; ints[4] = s->nz2r;
  dbls[0] = s->drho; dbls[1] = s->dr; dbls[2] = s->rhomax; dbls[3] = s->cutmax;
  return 0;
}

int orc_eam_tables(orc_sim *s, double *frho_spline, double *rhor_spline, double *z2r_spline,
                   int *t2frho, int *t2rhor, int *t2z2r) {
  if (s->pstyle != PS_EAM || !s->frho_spline) return fail(s, "eam not initialised");
  memcpy(frho_spline, s->frho_spline, sizeof(double) * (size_t)s->nfrho * (s->nrho + 1) * 7);
  memcpy(rhor_spline, s->rhor_spline, sizeof(double) * (size_t)s->nrhor * (s->nr + 1) * 7);
  memcpy(z2r_spline, s->z2r_spline, sizeof(double) * (size_t)s->nz2r * (s->nr + 1) * 7);
  int nt = s->ntypes;
  for (int i = 1; i <= nt; i++) {
    t2frho[i - 1] = s->type2frho[i];
    for (int j = 1; j <= nt; j++) {
      t2rhor[(i - 1) * nt + j - 1] = s->type2rhor[i][j];
      t2z2r[(i - 1) * nt + j - 1] = s->type2z2r[i][j];
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* domain, comm, neighbor                                              */

/* Domain::pbc for an orthogonal periodic box (src/domain.cpp:478-560) */
static void domain_pbc(orc_sim *s) {
  for (int i = 0; i < s->nlocal; i++)
    for (int d = 0; d < 3; d++) {
      double *x = s->x + 3 * i + d;
      if (*x < s->boxlo[d]) {
        *x += s->prd[d];
        s->image[3 * i + d]--;
      }
      if (*x >= s->boxhi[d]) {
        *x -= s->prd[d];
        *x = MAX(*x, s->boxlo[d]);
        s->image[3 * i + d]++;
      }
    }
}

/* CommBrick::setup for one process and a periodic box: two swaps per
   dimension, slabs [-BIG, lo+cutghost] with pbc +1 and [hi-cutghost, BIG]
   with pbc -1 (src/comm_brick.cpp:151-398) */
static int comm_setup(orc_sim *s) {
  double cutghost = s->cutneighmax;
  for (int d = 0; d < 3; d++) {
    int maxneed = (int)(cutghost * 1 / s->prd[d]) + 1;
    if (maxneed != 1)
      return fail(s, "box edge %g is not larger than the ghost cutoff %g", s->prd[d], cutghost);
  }
  s->nswap = 6;
  int iswap = 0;
  for (int d = 0; d < 3; d++)
    for (int ineed = 0; ineed < 2; ineed++) {
      s->pbc[iswap][0] = s->pbc[iswap][1] = s->pbc[iswap][2] = 0;
      if (ineed % 2 == 0) {
        s->slablo[iswap] = -BIG;
        s->slabhi[iswap] = s->boxlo[d] + cutghost;
        s->pbc[iswap][d] = 1;
      } else {
        s->slablo[iswap] = s->boxhi[d] - cutghost;
        s->slabhi[iswap] = BIG;
        s->pbc[iswap][d] = -1;
      }
      iswap++;
    }
  return 0;
}

/* CommBrick::borders + AtomVecAtomic::pack_border/unpack_border
   (src/comm_brick.cpp:696-864, src/atom_vec_atomic.cpp:268-311,392) */
static void comm_borders(orc_sim *s) {
  int iswap = 0;
  s->nghost = 0;
  for (int d = 0; d < 3; d++) {
    int nfirst = 0, nlast = 0;
    for (int ineed = 0; ineed < 2; ineed++) {
      double lo = s->slablo[iswap], hi = s->slabhi[iswap];
      if (ineed % 2 == 0) {
        nfirst = nlast;
        nlast = s->nlocal + s->nghost;
      }
      ilist_t *sl = &s->sendlist[iswap];
      sl->n = 0;
      for (int i = nfirst; i < nlast; i++)
        if (s->x[3 * i + d] >= lo && s->x[3 * i + d] <= hi) il_push(sl, i);
      int nsend = sl->n;
      int first = s->nlocal + s->nghost;
      grow_atoms(s, first + nsend + 1);
      double dx = s->pbc[iswap][0] * s->prd[0];
      double dy = s->pbc[iswap][1] * s->prd[1];
      double dz = s->pbc[iswap][2] * s->prd[2];
      for (int k = 0; k < nsend; k++) {
        int j = sl->list[k], g = first + k;
        s->x[3 * g] = s->x[3 * j] + dx;
        s->x[3 * g + 1] = s->x[3 * j + 1] + dy;
        s->x[3 * g + 2] = s->x[3 * j + 2] + dz;
        s->tag[g] = s->tag[j];
        s->type[g] = s->type[j];
        /* bookkeeping for list export: owning local atom and image */
        int owner = j < s->nlocal ? j : s->gowner[j];
        int gi = g;
        s->gowner[gi] = owner;
        for (int c = 0; c < 3; c++)
          s->gimg[3 * gi + c] = (j < s->nlocal ? 0 : s->gimg[3 * j + c]) + s->pbc[iswap][c];
      }
      s->firstrecv[iswap] = first;
      s->recvnum[iswap] = nsend;
      s->nghost += nsend;
      iswap++;
    }
  }
}

/* CommBrick::forward_comm + pack_comm (src/comm_brick.cpp:444-506,
   src/atom_vec_atomic.cpp:105-137) */
static void comm_forward(orc_sim *s) {
  for (int iswap = 0; iswap < s->nswap; iswap++) {
    double dx = s->pbc[iswap][0] * s->prd[0];
    double dy = s->pbc[iswap][1] * s->prd[1];
    double dz = s->pbc[iswap][2] * s->prd[2];
    const ilist_t *sl = &s->sendlist[iswap];
    int first = s->firstrecv[iswap];
    for (int k = 0; k < sl->n; k++) {
      int j = sl->list[k], g = first + k;
      s->x[3 * g] = s->x[3 * j] + dx;
      s->x[3 * g + 1] = s->x[3 * j + 1] + dy;
      s->x[3 * g + 2] = s->x[3 * j + 2] + dz;
    }
  }
}

/* CommBrick::reverse_comm of f (src/comm_brick.cpp:513-560) */
static void comm_reverse(orc_sim *s, double *a, int stride) {
  for (int iswap = s->nswap - 1; iswap >= 0; iswap--) {
    const ilist_t *sl = &s->sendlist[iswap];
    int first = s->firstrecv[iswap];
    for (int k = 0; k < sl->n; k++)
      for (int c = 0; c < stride; c++)
        a[(size_t)stride * sl->list[k] + c] += a[(size_t)stride * (first + k) + c];
  }
}

/* forward_comm_pair of fp (src/MANYBODY/pair_eam.cpp:232,809-831) */
static void comm_forward_scalar(orc_sim *s, double *a) {
  for (int iswap = 0; iswap < s->nswap; iswap++) {
    const ilist_t *sl = &s->sendlist[iswap];
    int first = s->firstrecv[iswap];
    for (int k = 0; k < sl->n; k++) a[first + k] = a[sl->list[k]];
  }
}

static double bin_distance(orc_sim *s, int i, int j, int k) {
  double delx, dely, delz;
  if (i > 0) delx = (i - 1) * s->binsizex;
  else if (i == 0) delx = 0.0;
  else delx = (i + 1) * s->binsizex;
  if (j > 0) dely = (j - 1) * s->binsizey;
  else if (j == 0) dely = 0.0;
  else dely = (j + 1) * s->binsizey;
  if (k > 0) delz = (k - 1) * s->binsizez;
  else if (k == 0) delz = 0.0;
  else delz = (k + 1) * s->binsizez;
  return delx * delx + dely * dely + delz * delz;
}

/* Neighbor::init cutoffs (src/neighbor.cpp:255-279) */
static void neigh_init(orc_sim *s) {
  s->cutneighmax = 0.0;
  for (int i = 1; i <= s->ntypes; i++)
    for (int j = 1; j <= s->ntypes; j++) {
      double cutoff = sqrt(s->cutsq[i][j]);
      double delta = cutoff > 0.0 ? s->skin : 0.0;
      double cut = cutoff + delta;
      s->cutneighsq[i][j] = cut * cut;
      s->cutneighmax = MAX(s->cutneighmax, cut);
    }
  s->cutneighmaxsq = s->cutneighmax * s->cutneighmax;
  s->triggersq = 0.25 * s->skin * s->skin; /* :239 */
}

/* Neighbor::setup_bins + stencil_half_bin_3d_newton
   (src/neighbor.cpp:1538-1702, src/neigh_stencil.cpp:143-158) */
static void setup_bins(orc_sim *s) {
  double cutghost = s->cutneighmax;
  double bsubboxlo[3], bsubboxhi[3], bbox[3];
  for (int d = 0; d < 3; d++) {
    bsubboxlo[d] = s->boxlo[d] - cutghost;
    bsubboxhi[d] = s->boxhi[d] + cutghost;
    bbox[d] = s->boxhi[d] - s->boxlo[d];
  }
  double binsize_optimal = 0.5 * s->cutneighmax;
  if (binsize_optimal == 0.0) binsize_optimal = bbox[0];
  double binsizeinv = 1.0 / binsize_optimal;
  s->nbinx = (int)(bbox[0] * binsizeinv);
  s->nbiny = (int)(bbox[1] * binsizeinv);
  s->nbinz = (int)(bbox[2] * binsizeinv);
  if (s->nbinx == 0) s->nbinx = 1;
  if (s->nbiny == 0) s->nbiny = 1;
  if (s->nbinz == 0) s->nbinz = 1;
  s->binsizex = bbox[0] / s->nbinx;
  s->binsizey = bbox[1] / s->nbiny;
  s->binsizez = bbox[2] / s->nbinz;
  s->bininvx = 1.0 / s->binsizex;
  s->bininvy = 1.0 / s->binsizey;
  s->bininvz = 1.0 / s->binsizez;
  int lo[3], hi[3];
  double inv[3] = {s->bininvx, s->bininvy, s->bininvz};
  for (int d = 0; d < 3; d++) {
    double coord = bsubboxlo[d] - SMALL * bbox[d];
    lo[d] = (int)((coord - s->boxlo[d]) * inv[d]);
    if (coord < s->boxlo[d]) lo[d] = lo[d] - 1;
    coord = bsubboxhi[d] + SMALL * bbox[d];
    hi[d] = (int)((coord - s->boxlo[d]) * inv[d]);
    lo[d] -= 1;
    hi[d] += 1;
  }
  s->mbinxlo = lo[0];
  s->mbinylo = lo[1];
  s->mbinzlo = lo[2];
  s->mbinx = hi[0] - lo[0] + 1;
  s->mbiny = hi[1] - lo[1] + 1;
  s->mbinz = hi[2] - lo[2] + 1;
  s->mbins = s->mbinx * s->mbiny * s->mbinz;
  s->binhead = (int *)xrealloc(s->binhead, sizeof(int) * (size_t)s->mbins);
  int sx = (int)(s->cutneighmax * s->bininvx);
  if (sx * s->binsizex < s->cutneighmax) sx++;
  int sy = (int)(s->cutneighmax * s->bininvy);
  if (sy * s->binsizey < s->cutneighmax) sy++;
  int sz = (int)(s->cutneighmax * s->bininvz);
  if (sz * s->binsizez < s->cutneighmax) sz++;
  int smax = (2 * sx + 1) * (2 * sy + 1) * (2 * sz + 1);
  s->stencil = (int *)xrealloc(s->stencil, sizeof(int) * (size_t)smax);
  s->nstencil = 0;
  for (int k = 0; k <= sz; k++)
    for (int j = -sy; j <= sy; j++)
      for (int i = -sx; i <= sx; i++)
        if (k > 0 || j > 0 || (j == 0 && i > 0))
          if (bin_distance(s, i, j, k) < s->cutneighmaxsq)
            s->stencil[s->nstencil++] = k * s->mbiny * s->mbinx + j * s->mbinx + i;
}

/* Neighbor::coord2bin (src/neighbor.cpp:1918-1947) */
static int coord2bin(const orc_sim *s, const double *x) {
  int ix, iy, iz;
  if (x[0] >= s->boxhi[0]) ix = (int)((x[0] - s->boxhi[0]) * s->bininvx) + s->nbinx;
  else if (x[0] >= s->boxlo[0]) {
    ix = (int)((x[0] - s->boxlo[0]) * s->bininvx);
    ix = MIN(ix, s->nbinx - 1);
  } else ix = (int)((x[0] - s->boxlo[0]) * s->bininvx) - 1;
  if (x[1] >= s->boxhi[1]) iy = (int)((x[1] - s->boxhi[1]) * s->bininvy) + s->nbiny;
  else if (x[1] >= s->boxlo[1]) {
    iy = (int)((x[1] - s->boxlo[1]) * s->bininvy);
    iy = MIN(iy, s->nbiny - 1);
  } else iy = (int)((x[1] - s->boxlo[1]) * s->bininvy) - 1;
  if (x[2] >= s->boxhi[2]) iz = (int)((x[2] - s->boxhi[2]) * s->bininvz) + s->nbinz;
  else if (x[2] >= s->boxlo[2]) {
    iz = (int)((x[2] - s->boxlo[2]) * s->bininvz);
    iz = MIN(iz, s->nbinz - 1);
  } else iz = (int)((x[2] - s->boxlo[2]) * s->bininvz) - 1;
  return (iz - s->mbinzlo) * s->mbiny * s->mbinx + (iy - s->mbinylo) * s->mbinx + (ix - s->mbinxlo);
}

/* Neighbor::bin_atoms: reverse order so each bin's linked list is in
   ascending index order with ghosts at the end (src/neighbor.cpp:1868-1904) */
static void bin_atoms(orc_sim *s) {
  for (int i = 0; i < s->mbins; i++) s->binhead[i] = -1;
  int nall = s->nlocal + s->nghost;
  for (int i = nall - 1; i >= 0; i--) {
    int ibin = coord2bin(s, s->x + 3 * i);
    s->bins[i] = s->binhead[ibin];
    s->binhead[ibin] = i;
  }
}

/* Neighbor::half_bin_newton for atomic systems (src/neigh_half_bin.cpp:285-419) */
static void half_bin_newton_range(orc_sim *s, int i0, int i1, ilist_t *page, long long *off) {
  const double *x = s->x;
  int nlocal = s->nlocal;
  for (int i = i0; i < i1; i++) {
    off[i - i0] = page->n;
    int n0 = page->n;
    int itype = s->type[i];
    double xtmp = x[3 * i], ytmp = x[3 * i + 1], ztmp = x[3 * i + 2];
    for (int j = s->bins[i]; j >= 0; j = s->bins[j]) {
      if (j >= nlocal) {
        if (x[3 * j + 2] < ztmp) continue;
        if (x[3 * j + 2] == ztmp) {
          if (x[3 * j + 1] < ytmp) continue;
          if (x[3 * j + 1] == ytmp && x[3 * j] < xtmp) continue;
        }
      }
      int jtype = s->type[j];
      double delx = xtmp - x[3 * j], dely = ytmp - x[3 * j + 1], delz = ztmp - x[3 * j + 2];
      double rsq = delx * delx + dely * dely + delz * delz;
      if (rsq <= s->cutneighsq[itype][jtype]) il_push(page, j);
    }
    int ibin = coord2bin(s, x + 3 * i);
    for (int k = 0; k < s->nstencil; k++)
      for (int j = s->binhead[ibin + s->stencil[k]]; j >= 0; j = s->bins[j]) {
        int jtype = s->type[j];
        double delx = xtmp - x[3 * j], dely = ytmp - x[3 * j + 1], delz = ztmp - x[3 * j + 2];
        double rsq = delx * delx + dely * dely + delz * delz;
        if (rsq <= s->cutneighsq[itype][jtype]) il_push(page, j);
      }
    s->numneigh[i] = page->n - n0;
  }
}

/* Neighbor::build (src/neighbor.cpp:1380-1461) */
static void neigh_build(orc_sim *s) {
  s->ago = 0;
  s->ncalls++;
  if (s->dist_check) {
    s->xhold = (double *)xrealloc(s->xhold, sizeof(double) * 3 * (size_t)s->nmax);
    memcpy(s->xhold, s->x, sizeof(double) * 3 * (size_t)s->nlocal);
  }
  bin_atoms(s);
  int n = s->nlocal;
  s->numneigh = (int *)xrealloc(s->numneigh, sizeof(int) * (size_t)(n + 1));
  s->firstneigh = (int **)xrealloc(s->firstneigh, sizeof(int *) * (size_t)(n + 1));
  int nt = s->nthreads;
  if (s->nbuf < nt) {
    s->neighbuf = (ilist_t *)xrealloc(s->neighbuf, sizeof(ilist_t) * (size_t)nt);
    for (int t = s->nbuf; t < nt; t++) memset(&s->neighbuf[t], 0, sizeof(ilist_t));
    s->nbuf = nt;
  }
  long long *off = (long long *)malloc(sizeof(long long) * (size_t)(n + 1));
#pragma omp parallel num_threads(nt) if (nt > 1)
  {
    int t = 0, T = 1;
#ifdef _OPENMP
    t = omp_get_thread_num();
    T = omp_get_num_threads();
#endif
    int i0 = (int)((long long)n * t / T), i1 = (int)((long long)n * (t + 1) / T);
    s->neighbuf[t].n = 0;
    half_bin_newton_range(s, i0, i1, &s->neighbuf[t], off + i0);
#pragma omp barrier
    for (int i = i0; i < i1; i++) s->firstneigh[i] = s->neighbuf[t].list + off[i];
  }
  free(off);
}

/* Neighbor::decide + check_distance (src/neighbor.cpp:1294-1372) */
static int neigh_decide(orc_sim *s) {
  s->ago++;
  if (s->ago >= s->delay && s->ago % s->every == 0) {
    if (s->dist_check == 0) return 1;
    int flag = 0;
    for (int i = 0; i < s->nlocal; i++) {
      double delx = s->x[3 * i] - s->xhold[3 * i];
      double dely = s->x[3 * i + 1] - s->xhold[3 * i + 1];
      double delz = s->x[3 * i + 2] - s->xhold[3 * i + 2];
      double rsq = delx * delx + dely * dely + delz * delz;
      if (rsq > s->triggersq) flag = 1;
    }
    if (flag && s->ago == MAX(s->every, s->delay)) s->ndanger++;
    return flag;
  }
  return 0;
}

/* Atom::setup_sort_bins + Atom::sort (src/atom.cpp:1575-1742): stable
   permutation of local atoms into bins of size half the neighbor cutoff */
static void atom_sort(orc_sim *s) {
  s->nextsort = (s->ntimestep / s->sortfreq) * s->sortfreq + s->sortfreq;
  double binsize = 0.5 * s->cutneighmax;
  double bininv = 1.0 / binsize;
  int nb[3];
  double binv[3];
  for (int d = 0; d < 3; d++) {
    nb[d] = (int)((s->boxhi[d] - s->boxlo[d]) * bininv);
    if (nb[d] == 0) nb[d] = 1;
    binv[d] = nb[d] / (s->boxhi[d] - s->boxlo[d]);
  }
  int nbins = nb[0] * nb[1] * nb[2];
  if (nbins == 1) return;
  int n = s->nlocal;
  int *head = (int *)malloc(sizeof(int) * (size_t)nbins);
  int *next = (int *)malloc(sizeof(int) * (size_t)n);
  int *perm = (int *)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < nbins; i++) head[i] = -1;
  for (int i = n - 1; i >= 0; i--) {
    int ix = (int)((s->x[3 * i] - s->boxlo[0]) * binv[0]);
    int iy = (int)((s->x[3 * i + 1] - s->boxlo[1]) * binv[1]);
    int iz = (int)((s->x[3 * i + 2] - s->boxlo[2]) * binv[2]);
    ix = MIN(MAX(ix, 0), nb[0] - 1);
    iy = MIN(MAX(iy, 0), nb[1] - 1);
    iz = MIN(MAX(iz, 0), nb[2] - 1);
    int ibin = iz * nb[1] * nb[0] + iy * nb[0] + ix;
    next[i] = head[ibin];
    head[ibin] = i;
  }
  int m = 0;
  for (int b = 0; b < nbins; b++)
    for (int i = head[b]; i >= 0; i = next[i]) perm[m++] = i;
  /* apply permutation: new[i] = old[perm[i]] */
  double *x = (double *)malloc(sizeof(double) * 3 * (size_t)n);
  double *v = (double *)malloc(sizeof(double) * 3 * (size_t)n);
  double *f = (double *)malloc(sizeof(double) * 3 * (size_t)n);
  int *ty = (int *)malloc(sizeof(int) * (size_t)n);
  int *tg = (int *)malloc(sizeof(int) * (size_t)n);
  int *im = (int *)malloc(sizeof(int) * 3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    int o = perm[i];
    memcpy(x + 3 * i, s->x + 3 * o, 3 * sizeof(double));
    memcpy(v + 3 * i, s->v + 3 * o, 3 * sizeof(double));
    memcpy(f + 3 * i, s->f + 3 * o, 3 * sizeof(double));
    memcpy(im + 3 * i, s->image + 3 * o, 3 * sizeof(int));
    ty[i] = s->type[o];
    tg[i] = s->tag[o];
  }
  memcpy(s->x, x, sizeof(double) * 3 * (size_t)n);
  memcpy(s->v, v, sizeof(double) * 3 * (size_t)n);
  memcpy(s->f, f, sizeof(double) * 3 * (size_t)n);
  memcpy(s->image, im, sizeof(int) * 3 * (size_t)n);
  memcpy(s->type, ty, sizeof(int) * (size_t)n);
  memcpy(s->tag, tg, sizeof(int) * (size_t)n);
  free(x); free(v); free(f); free(ty); free(tg); free(im);
  free(head); free(next); free(perm);
}

/* ------------------------------------------------------------------ */
/* pair computes                                                       */

/* Pair::ev_setup (src/pair.cpp:679-742) */
static void ev_setup(orc_sim *s, int eflag, int vflag) {
  s->evflag = 1;
  s->eflag_global = eflag % 2;
  s->eflag_atom = eflag / 2;
  s->vflag_global = vflag % 4;
  s->vflag_atom = vflag / 4;
  int nall = s->nlocal + s->nghost;
  if (s->eflag_global) s->eng_vdwl = 0.0;
  if (s->vflag_global)
    for (int i = 0; i < 6; i++) s->virial[i] = 0.0;
  if (s->eflag_atom) memset(s->eatom, 0, sizeof(double) * (size_t)nall);
  if (s->vflag_atom) memset(s->vatom, 0, sizeof(double) * 6 * (size_t)nall);
  if (s->vflag_global == 2) {
    s->vflag_fdotr = 1;
    s->vflag_global = 0;
    if (s->vflag_atom == 0 && eflag == 0) s->evflag = 0;
  } else
    s->vflag_fdotr = 0;
}

/* Pair::ev_tally with newton_pair = 1 (src/pair.cpp:769-855) */
typedef struct {
  double eng, vir[6];
} evacc;

static inline void ev_tally(orc_sim *s, evacc *a, double *eatom, double *vatom, int i, int j,
                            double evdwl, double fpair, double delx, double dely, double delz) {
  if (s->eflag_global) a->eng += evdwl;
  if (s->eflag_atom) {
    double epairhalf = 0.5 * evdwl;
    eatom[i] += epairhalf;
    eatom[j] += epairhalf;
  }
  if (s->vflag_global || s->vflag_atom) {
    double v[6];
    v[0] = delx * delx * fpair;
    v[1] = dely * dely * fpair;
    v[2] = delz * delz * fpair;
    v[3] = delx * dely * fpair;
    v[4] = delx * delz * fpair;
    v[5] = dely * delz * fpair;
    if (s->vflag_global)
      for (int k = 0; k < 6; k++) a->vir[k] += v[k];
    if (s->vflag_atom)
      for (int k = 0; k < 6; k++) {
        vatom[6 * i + k] += 0.5 * v[k];
        vatom[6 * j + k] += 0.5 * v[k];
      }
  }
}

/* Pair::virial_fdotr_compute over nlocal+nghost (src/pair.cpp:1402-1450) */
static void virial_fdotr(orc_sim *s) {
  int nall = s->nlocal + s->nghost;
  for (int i = 0; i < nall; i++) {
    const double *f = s->f + 3 * i, *x = s->x + 3 * i;
    s->virial[0] += f[0] * x[0];
    s->virial[1] += f[1] * x[1];
    s->virial[2] += f[2] * x[2];
    s->virial[3] += f[1] * x[0];
    s->virial[4] += f[2] * x[0];
    s->virial[5] += f[2] * x[1];
  }
  s->vflag_fdotr = 0;
}

/* per-thread private arrays, reduced in thread order
   (src/USER-OMP/thr_omp.cpp:149-214) */
typedef struct {
  double *f, *rho, *eatom, *vatom;
  evacc acc;
} thrbuf;

static thrbuf *thr_alloc(orc_sim *s, int nt, int need_rho) {
  int nall = s->nlocal + s->nghost;
  thrbuf *b = (thrbuf *)calloc((size_t)nt, sizeof(thrbuf));
  for (int t = 0; t < nt; t++) {
    b[t].f = (double *)calloc(3 * (size_t)nall, sizeof(double));
    if (need_rho) b[t].rho = (double *)calloc((size_t)nall, sizeof(double));
    if (s->eflag_atom) b[t].eatom = (double *)calloc((size_t)nall, sizeof(double));
    if (s->vflag_atom) b[t].vatom = (double *)calloc(6 * (size_t)nall, sizeof(double));
  }
  return b;
}

static void thr_free(thrbuf *b, int nt) {
  for (int t = 0; t < nt; t++) {
    free(b[t].f); free(b[t].rho); free(b[t].eatom); free(b[t].vatom);
  }
  free(b);
}

static void thr_reduce(orc_sim *s, thrbuf *b, int nt) {
  int nall = s->nlocal + s->nghost;
  for (int t = 0; t < nt; t++) {
    for (size_t k = 0; k < 3 * (size_t)nall; k++) s->f[k] += b[t].f[k];
    if (s->eflag_global) s->eng_vdwl += b[t].acc.eng;
    if (s->vflag_global)
      for (int k = 0; k < 6; k++) s->virial[k] += b[t].acc.vir[k];
    if (s->eflag_atom)
      for (int k = 0; k < nall; k++) s->eatom[k] += b[t].eatom[k];
    if (s->vflag_atom)
      for (size_t k = 0; k < 6 * (size_t)nall; k++) s->vatom[k] += b[t].vatom[k];
  }
}

/* PairLJCut::compute with newton_pair on (src/pair_lj_cut.cpp:68-141) */
static void lj_range(orc_sim *s, int i0, int i1, double *f, evacc *a, double *eatom,
                     double *vatom) {
  const double *x = s->x;
  for (int i = i0; i < i1; i++) {
    double xtmp = x[3 * i], ytmp = x[3 * i + 1], ztmp = x[3 * i + 2];
    int itype = s->type[i];
    const int *jlist = s->firstneigh[i];
    int jnum = s->numneigh[i];
    for (int jj = 0; jj < jnum; jj++) {
      int j = jlist[jj];
      double delx = xtmp - x[3 * j], dely = ytmp - x[3 * j + 1], delz = ztmp - x[3 * j + 2];
      double rsq = delx * delx + dely * dely + delz * delz;
      int jtype = s->type[j];
      if (rsq < s->cutsq[itype][jtype]) {
        double r2inv = 1.0 / rsq;
        double r6inv = r2inv * r2inv * r2inv;
        double forcelj = r6inv * (s->lj1[itype][jtype] * r6inv - s->lj2[itype][jtype]);
        double fpair = 1.0 * forcelj * r2inv;
        f[3 * i] += delx * fpair;
        f[3 * i + 1] += dely * fpair;
        f[3 * i + 2] += delz * fpair;
        f[3 * j] -= delx * fpair;
        f[3 * j + 1] -= dely * fpair;
        f[3 * j + 2] -= delz * fpair;
        double evdwl = 0.0;
        if (s->eflag_global || s->eflag_atom) {
          evdwl = r6inv * (s->lj3[itype][jtype] * r6inv - s->lj4[itype][jtype]) -
                  s->offset[itype][jtype];
          evdwl *= 1.0;
        }
        if (s->evflag) ev_tally(s, a, eatom, vatom, i, j, evdwl, fpair, delx, dely, delz);
      }
    }
  }
}

static void pair_lj_compute(orc_sim *s, int eflag, int vflag) {
  if (eflag || vflag) ev_setup(s, eflag, vflag);
  else s->evflag = s->vflag_fdotr = s->eflag_global = s->eflag_atom = s->vflag_global =
           s->vflag_atom = 0;
  int nt = s->nthreads, n = s->nlocal;
  if (nt <= 1) {
    evacc a = {0.0, {0, 0, 0, 0, 0, 0}};
    lj_range(s, 0, n, s->f, &a, s->eatom, s->vatom);
    if (s->eflag_global) s->eng_vdwl += a.eng;
    if (s->vflag_global)
      for (int k = 0; k < 6; k++) s->virial[k] += a.vir[k];
  } else {
    thrbuf *b = thr_alloc(s, nt, 0);
#pragma omp parallel num_threads(nt)
    {
      int t = 0, T = 1;
#ifdef _OPENMP
      t = omp_get_thread_num();
      T = omp_get_num_threads();
#endif
      int i0 = (int)((long long)n * t / T), i1 = (int)((long long)n * (t + 1) / T);
      lj_range(s, i0, i1, b[t].f, &b[t].acc, b[t].eatom, b[t].vatom);
    }
    thr_reduce(s, b, nt);
    thr_free(b, nt);
  }
  if (s->vflag_fdotr) virial_fdotr(s);
}

/* PairEAM::compute, three passes with newton on
   (src/MANYBODY/pair_eam.cpp:125-306) */
static void eam_rho_range(orc_sim *s, int i0, int i1, double *rho) {
  const double *x = s->x;
  int nr = s->nr;
  for (int i = i0; i < i1; i++) {
    double xtmp = x[3 * i], ytmp = x[3 * i + 1], ztmp = x[3 * i + 2];
    int itype = s->type[i];
    const int *jlist = s->firstneigh[i];
    int jnum = s->numneigh[i];
    for (int jj = 0; jj < jnum; jj++) {
      int j = jlist[jj];
      double delx = xtmp - x[3 * j], dely = ytmp - x[3 * j + 1], delz = ztmp - x[3 * j + 2];
      double rsq = delx * delx + dely * dely + delz * delz;
      if (rsq < s->cutforcesq) {
        int jtype = s->type[j];
        double p = sqrt(rsq) * s->rdr + 1.0;
        int m = (int)p;
        m = MIN(m, nr - 1);
        p -= m;
        p = MIN(p, 1.0);
        const double *coeff = s->rhor_spline + ((size_t)s->type2rhor[jtype][itype] * (nr + 1) + m) * 7;
        rho[i] += ((coeff[3] * p + coeff[4]) * p + coeff[5]) * p + coeff[6];
        coeff = s->rhor_spline + ((size_t)s->type2rhor[itype][jtype] * (nr + 1) + m) * 7;
        rho[j] += ((coeff[3] * p + coeff[4]) * p + coeff[5]) * p + coeff[6];
      }
    }
  }
}

static void eam_force_range(orc_sim *s, int i0, int i1, double *f, evacc *a, double *eatom,
                            double *vatom) {
  const double *x = s->x;
  int nr = s->nr;
  for (int i = i0; i < i1; i++) {
    double xtmp = x[3 * i], ytmp = x[3 * i + 1], ztmp = x[3 * i + 2];
    int itype = s->type[i];
    const int *jlist = s->firstneigh[i];
    int jnum = s->numneigh[i];
    for (int jj = 0; jj < jnum; jj++) {
      int j = jlist[jj];
      double delx = xtmp - x[3 * j], dely = ytmp - x[3 * j + 1], delz = ztmp - x[3 * j + 2];
      double rsq = delx * delx + dely * dely + delz * delz;
      if (rsq < s->cutforcesq) {
        int jtype = s->type[j];
        double r = sqrt(rsq);
        double p = r * s->rdr + 1.0;
        int m = (int)p;
        m = MIN(m, nr - 1);
        p -= m;
        p = MIN(p, 1.0);
        const double *coeff;
        coeff = s->rhor_spline + ((size_t)s->type2rhor[itype][jtype] * (nr + 1) + m) * 7;
        double rhoip = (coeff[0] * p + coeff[1]) * p + coeff[2];
        coeff = s->rhor_spline + ((size_t)s->type2rhor[jtype][itype] * (nr + 1) + m) * 7;
        double rhojp = (coeff[0] * p + coeff[1]) * p + coeff[2];
        coeff = s->z2r_spline + ((size_t)s->type2z2r[itype][jtype] * (nr + 1) + m) * 7;
        double z2p = (coeff[0] * p + coeff[1]) * p + coeff[2];
        double z2 = ((coeff[3] * p + coeff[4]) * p + coeff[5]) * p + coeff[6];
        double recip = 1.0 / r;
        double phi = z2 * recip;
        double phip = z2p * recip - phi * recip;
        double psip = s->fp[i] * rhojp + s->fp[j] * rhoip + phip;
        double fpair = -psip * recip;
        f[3 * i] += delx * fpair;
        f[3 * i + 1] += dely * fpair;
        f[3 * i + 2] += delz * fpair;
        f[3 * j] -= delx * fpair;
        f[3 * j + 1] -= dely * fpair;
        f[3 * j + 2] -= delz * fpair;
        double evdwl = (s->eflag_global || s->eflag_atom) ? phi : 0.0;
        if (s->evflag) ev_tally(s, a, eatom, vatom, i, j, evdwl, fpair, delx, dely, delz);
      }
    }
  }
}

static void pair_eam_compute(orc_sim *s, int eflag, int vflag) {
  if (eflag || vflag) ev_setup(s, eflag, vflag);
  else s->evflag = s->vflag_fdotr = s->eflag_global = s->eflag_atom = s->vflag_global =
           s->vflag_atom = 0;
  int nall = s->nlocal + s->nghost, n = s->nlocal, nt = s->nthreads;
  for (int i = 0; i < nall; i++) s->rho[i] = 0.0;
  if (nt <= 1) {
    eam_rho_range(s, 0, n, s->rho);
  } else {
    thrbuf *b = thr_alloc(s, nt, 1);
#pragma omp parallel num_threads(nt)
    {
      int t = 0, T = 1;
#ifdef _OPENMP
      t = omp_get_thread_num();
      T = omp_get_num_threads();
#endif
      int i0 = (int)((long long)n * t / T), i1 = (int)((long long)n * (t + 1) / T);
      eam_rho_range(s, i0, i1, b[t].rho);
    }
    for (int t = 0; t < nt; t++)
      for (int k = 0; k < nall; k++) s->rho[k] += b[t].rho[k];
    thr_free(b, nt);
  }
  comm_reverse(s, s->rho, 1);
  int nrho = s->nrho;
  for (int i = 0; i < n; i++) {
    double p = s->rho[i] * s->rdrho + 1.0;
    int m = (int)p;
    m = MAX(1, MIN(m, nrho - 1));
    p -= m;
    p = MIN(p, 1.0);
    const double *coeff = s->frho_spline + ((size_t)s->type2frho[s->type[i]] * (nrho + 1) + m) * 7;
    s->fp[i] = (coeff[0] * p + coeff[1]) * p + coeff[2];
    if (eflag) {
      double phi = ((coeff[3] * p + coeff[4]) * p + coeff[5]) * p + coeff[6];
      if (s->rho[i] > s->rhomax) phi += s->fp[i] * (s->rho[i] - s->rhomax);
      if (s->eflag_global) s->eng_vdwl += phi;
      if (s->eflag_atom) s->eatom[i] += phi;
    }
  }
  comm_forward_scalar(s, s->fp);
  if (nt <= 1) {
    evacc a = {0.0, {0, 0, 0, 0, 0, 0}};
    eam_force_range(s, 0, n, s->f, &a, s->eatom, s->vatom);
    if (s->eflag_global) s->eng_vdwl += a.eng;
    if (s->vflag_global)
      for (int k = 0; k < 6; k++) s->virial[k] += a.vir[k];
  } else {
    thrbuf *b = thr_alloc(s, nt, 0);
#pragma omp parallel num_threads(nt)
    {
      int t = 0, T = 1;
#ifdef _OPENMP
      t = omp_get_thread_num();
      T = omp_get_num_threads();
#endif
      int i0 = (int)((long long)n * t / T), i1 = (int)((long long)n * (t + 1) / T);
      eam_force_range(s, i0, i1, b[t].f, &b[t].acc, b[t].eatom, b[t].vatom);
    }
    thr_reduce(s, b, nt);
    thr_free(b, nt);
  }
  if (s->vflag_fdotr) virial_fdotr(s);
}

static void force_clear(orc_sim *s) {
  memset(s->f, 0, sizeof(double) * 3 * (size_t)(s->nlocal + s->nghost));
}

static void pair_compute(orc_sim *s, int eflag, int vflag) {
  if (s->pstyle == PS_LJ) pair_lj_compute(s, eflag, vflag);
  else pair_eam_compute(s, eflag, vflag);
}

/* ------------------------------------------------------------------ */
/* integration and driver                                              */

/* FixNVE::initial_integrate / final_integrate (src/fix_nve.cpp:65-142),
   dtf = 0.5 dt ftm2v (:52-59) */
static void nve_initial(orc_sim *s) {
  double dtv = s->dt, dtf = 0.5 * s->dt * s->ftm2v;
  for (int i = 0; i < s->nlocal; i++) {
    double dtfm = dtf / s->mass[s->type[i]];
    double *v = s->v + 3 * i, *x = s->x + 3 * i;
    const double *f = s->f + 3 * i;
    v[0] += dtfm * f[0];
    v[1] += dtfm * f[1];
    v[2] += dtfm * f[2];
    x[0] += dtv * v[0];
    x[1] += dtv * v[1];
    x[2] += dtv * v[2];
  }
}

static void nve_final(orc_sim *s) {
  double dtf = 0.5 * s->dt * s->ftm2v;
  for (int i = 0; i < s->nlocal; i++) {
    double dtfm = dtf / s->mass[s->type[i]];
    double *v = s->v + 3 * i;
    const double *f = s->f + 3 * i;
    v[0] += dtfm * f[0];
    v[1] += dtfm * f[1];
    v[2] += dtfm * f[2];
  }
}

/* Thermo one-line output: Temp, E_pair, TotEng, Press
   (src/thermo.cpp:1581-1619, src/compute_pressure.cpp:177-207) */
static void thermo_row(orc_sim *s) {
  double t = temp_scalar(s);
  double dof = 3.0 * s->nlocal - 3.0;
  double natoms = s->nlocal;
  double pe = s->eng_vdwl;
  double epair = s->normflag ? pe / natoms : pe;
  double ke = t * 0.5 * dof * s->boltz;
  if (s->normflag) ke /= natoms;
  double inv_volume = 1.0 / (s->prd[0] * s->prd[1] * s->prd[2]);
  double press = (dof * s->boltz * t + s->virial[0] + s->virial[1] + s->virial[2]) / 3.0 *
                 inv_volume * s->nktv2p;
  s->temp_scalar = t;
  s->press_scalar = press;
  if (s->nrows == s->maxrows) {
    s->maxrows = s->maxrows ? 2 * s->maxrows : 16;
    s->rows = (double *)xrealloc(s->rows, sizeof(double) * 5 * (size_t)s->maxrows);
  }
  double *r = s->rows + 5 * s->nrows++;
  r[0] = (double)s->ntimestep;
  r[1] = t;
  r[2] = epair;
  r[3] = epair + ke;
  r[4] = press;
}

static int init_all(orc_sim *s) {
  if (!s->box_set) return fail(s, "box not set");
  if (s->pstyle == PS_LJ) {
    if (init_lj(s)) return -1;
  } else if (s->pstyle == PS_EAM) {
    if (init_eam(s)) return -1;
  } else
    return fail(s, "no pair style");
  for (int t = 1; t <= s->ntypes; t++)
    if (!(s->mass[t] > 0.0)) return fail(s, "mass not set for type %d", t);
  neigh_init(s);
  return comm_setup(s);
}

/* Verlet::setup (src/verlet.cpp:88-142) with eflag=1, vflag=2 at step 0 */
int orc_setup(orc_sim *s) {
  if (init_all(s)) return -1;
  s->ncalls = 0;
  s->ndanger = 0;
  s->nrows = 0;
  domain_pbc(s);
  setup_bins(s);
  if (s->sortfreq > 0) atom_sort(s);
  comm_borders(s);
  neigh_build(s);
  s->ncalls = 0;
  force_clear(s);
  pair_compute(s, 1, 2);
  comm_reverse(s, s->f, 3);
  thermo_row(s);
  s->setup_done = 1;
  return 0;
}

int orc_compute(orc_sim *s, int eflag, int vflag) {
  if (init_all(s)) return -1;
  domain_pbc(s);
  setup_bins(s);
  comm_borders(s);
  neigh_build(s);
  force_clear(s);
  pair_compute(s, eflag, vflag);
  /* per-atom tallies of ghosts folded into owners (reverse comm) */
  if (s->eflag_atom) comm_reverse(s, s->eatom, 1);
  if (s->vflag_atom) comm_reverse(s, s->vatom, 6);
  comm_reverse(s, s->f, 3);
  return 0;
}

/* Verlet::run (src/verlet.cpp:207-309) */
int orc_run(orc_sim *s, int nsteps) {
  if (!s->setup_done) return fail(s, "orc_setup not called");
  s->laststep = s->ntimestep + nsteps;
  for (int istep = 0; istep < nsteps; istep++) {
    s->ntimestep++;
    int out = (s->ntimestep == s->laststep) ||
              (s->thermo_every > 0 && s->ntimestep % s->thermo_every == 0);
    int eflag = out ? 1 : 0, vflag = out ? 2 : 0;
    nve_initial(s);
    if (neigh_decide(s) == 0) {
      comm_forward(s);
    } else {
      domain_pbc(s);
      if (s->sortfreq > 0 && s->ntimestep >= s->nextsort) atom_sort(s);
      comm_borders(s);
      neigh_build(s);
    }
    force_clear(s);
    pair_compute(s, eflag, vflag);
    comm_reverse(s, s->f, 3);
    nve_final(s);
    if (out) thermo_row(s);
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* accessors                                                           */

int orc_thermo_rows(orc_sim *s, double *out, int maxrows) {
  int n = MIN(maxrows, s->nrows);
  if (out) memcpy(out, s->rows, sizeof(double) * 5 * (size_t)n);
  return s->nrows;
}
int orc_nlocal(orc_sim *s) { return s->nlocal; }
int orc_nghost(orc_sim *s) { return s->nghost; }
int orc_ncalls(orc_sim *s) { return s->ncalls; }
int orc_ndanger(orc_sim *s) { return s->ndanger; }
long long orc_ntimestep(orc_sim *s) { return s->ntimestep; }
long long orc_neigh_total(orc_sim *s) {
  long long t = 0;
  for (int i = 0; i < s->nlocal; i++) t += s->numneigh[i];
  return t;
}
double orc_eng_vdwl(orc_sim *s) { return s->eng_vdwl; }
void orc_virial(orc_sim *s, double v[6]) { memcpy(v, s->virial, sizeof(s->virial)); }
double orc_temperature(orc_sim *s) { return temp_scalar(s); }
double orc_pressure(orc_sim *s) { return s->press_scalar; }
double orc_kinetic(orc_sim *s) {
  double dof = 3.0 * s->nlocal - 3.0;
  return temp_scalar(s) * 0.5 * dof * s->boltz;
}
void orc_get_x(orc_sim *s, double *x) { memcpy(x, s->x, sizeof(double) * 3 * (size_t)s->nlocal); }
void orc_get_v(orc_sim *s, double *v) { memcpy(v, s->v, sizeof(double) * 3 * (size_t)s->nlocal); }
void orc_get_f(orc_sim *s, double *f) { memcpy(f, s->f, sizeof(double) * 3 * (size_t)s->nlocal); }
void orc_get_tag(orc_sim *s, int *t) { memcpy(t, s->tag, sizeof(int) * (size_t)s->nlocal); }
void orc_get_type(orc_sim *s, int *t) { memcpy(t, s->type, sizeof(int) * (size_t)s->nlocal); }
void orc_get_image(orc_sim *s, int *im) { memcpy(im, s->image, sizeof(int) * 3 * (size_t)s->nlocal); }
void orc_get_rho_fp(orc_sim *s, double *rho, double *fp) {
  memcpy(rho, s->rho, sizeof(double) * (size_t)s->nlocal);
  memcpy(fp, s->fp, sizeof(double) * (size_t)s->nlocal);
}
void orc_get_eatom_vatom(orc_sim *s, double *eatom, double *vatom) {
  if (eatom) memcpy(eatom, s->eatom, sizeof(double) * (size_t)s->nlocal);
  if (vatom) memcpy(vatom, s->vatom, sizeof(double) * 6 * (size_t)s->nlocal);
}

long long orc_neigh_half(orc_sim *s, int *numneigh, int *jowner, int *jimage, long long cap) {
  long long m = 0;
  for (int i = 0; i < s->nlocal; i++) {
    if (numneigh) numneigh[i] = s->numneigh[i];
    for (int k = 0; k < s->numneigh[i]; k++) {
      int j = s->firstneigh[i][k];
      if (m < cap) {
        if (j < s->nlocal) {
          jowner[m] = j;
          jimage[m] = 13;
        } else {
          jowner[m] = s->gowner[j];
          const int *g = s->gimg + 3 * j;
          jimage[m] = (g[0] + 1) + 3 * (g[1] + 1) + 9 * (g[2] + 1);
        }
      }
      m++;
    }
  }
  return m;
}
