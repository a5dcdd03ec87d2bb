/*
 * md_oracle.h -- CPU oracle for the short-range MD step (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of the reference's serial CPU path
 * (LAMMPS "8 Aug 2014"): lattice creation, velocity create, periodic ghost
 * atoms (CommBrick::borders), binned half neighbor list with Newton
 * (Neighbor::half_bin_newton), pair_style lj/cut and eam / eam/alloy / eam/fs,
 * fix nve, the F.r virial and the thermo reductions.  It exists only so the
 * tests, the smoke check and the CPU-baseline leg of bench.py can check the
 * CUDA engine; the product never calls it.
 *
 * Parity pin: the reference cannot be built here without its own build
 * system (generated style headers), so the oracle is pinned against the
 * golden thermo logs and neighbor statistics shipped with the reference
 * (bench/log.1Feb14.{lj,eam}.fixed.linux.1) -- see tests/test_oracle_golden.py.
 */
#ifndef MD_ORACLE_H
#define MD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

/* units: 0 = lj, 1 = metal (src/update.cpp:118-166) */
orc_sim *orc_create(int unit_style);
void orc_destroy(orc_sim *s);
const char *orc_error(orc_sim *s);

void orc_set_threads(orc_sim *s, int nthreads);
void orc_set_timestep(orc_sim *s, double dt);
int  orc_set_box(orc_sim *s, const double lo[3], const double hi[3]);
int  orc_set_atoms(orc_sim *s, int n, int ntypes, const double *x, const double *v,
                   const int *type, const int *tag);
void orc_set_mass(orc_sim *s, int itype, double m);
/* neighbor skin bin + neigh_modify every/delay/check; sortfreq as atom_modify sort */
void orc_set_neighbor(orc_sim *s, double skin, int every, int delay, int check,
                      int sortfreq);
/* thermo output every N steps (0 = first and last only) */
void orc_set_thermo(orc_sim *s, int every);

/* pair_style lj/cut <cut_global>; pair_modify shift yes|no */
int orc_pair_lj_cut(orc_sim *s, double cut_global, int shift);
/* pair_coeff i j eps sigma [cut]  (cut < 0 -> global) */
int orc_pair_lj_coeff(orc_sim *s, int i, int j, double eps, double sigma, double cut);

/* pair_style eam: one funcfl file per type (file[itype-1]) */
int orc_pair_eam_funcfl(orc_sim *s, int nfiles, const char **files, const int *type2file);
/* pair_style eam/alloy (fs=0) or eam/fs (fs=1): map[itype-1] = element index or -1 */
int orc_pair_eam_setfl(orc_sim *s, const char *file, int fs, const int *map);

/* Verlet::setup: pbc, sort, borders, neighbor build, forces at step 0, thermo */
int orc_setup(orc_sim *s);
/* Verlet::run for n steps */
int orc_run(orc_sim *s, int nsteps);
/* force/energy/virial evaluation on current atoms (setup without output);
   vflag = 1 pairwise virial, 2 F.r virial */
int orc_compute(orc_sim *s, int eflag, int vflag);

/* thermo rows: step, temp, epair, etotal, press (5 doubles each) */
int orc_thermo_rows(orc_sim *s, double *out, int maxrows);

int orc_nlocal(orc_sim *s);
int orc_nghost(orc_sim *s);
int orc_ncalls(orc_sim *s);
int orc_ndanger(orc_sim *s);
long long orc_ntimestep(orc_sim *s);
long long orc_neigh_total(orc_sim *s);
double orc_eng_vdwl(orc_sim *s);
void orc_virial(orc_sim *s, double v[6]);
double orc_temperature(orc_sim *s);
double orc_pressure(orc_sim *s);
double orc_kinetic(orc_sim *s);

/* local atoms in the oracle's current index order */
void orc_get_x(orc_sim *s, double *x);
void orc_get_v(orc_sim *s, double *v);
void orc_get_f(orc_sim *s, double *f);
void orc_get_tag(orc_sim *s, int *tag);
void orc_get_type(orc_sim *s, int *type);
void orc_get_image(orc_sim *s, int *img);
void orc_get_rho_fp(orc_sim *s, double *rho, double *fp);
/* per-atom eatom (n) and vatom (n*6) after orc_compute with eflag/vflag atom */
void orc_get_eatom_vatom(orc_sim *s, double *eatom, double *vatom);

/* half neighbor list of local atoms: numneigh[n]; entries (index of the
   owning local atom, image code = (sx+1)+3(sy+1)+9(sz+1)) */
long long orc_neigh_half(orc_sim *s, int *numneigh, int *jowner, int *jimage,
                         long long cap);

/* EAM spline tables after init (7 coefficients per knot, LAMMPS layout) */
int orc_eam_info(orc_sim *s, int *ints /* nrho nr nfrho nrhor nz2r */,
                 double *dbls /* drho dr rhomax cutmax */);
int orc_eam_tables(orc_sim *s, double *frho_spline, double *rhor_spline,
                   double *z2r_spline, int *type2frho, int *type2rhor, int *type2z2r);

/* ---- input generators used by the checks ---- */
/* create_atoms on an fcc/sc/bcc lattice of nx*ny*nz unit cells, scale = lattice
   constant; returns atoms written (x[3n], tags 1..n in creation order) */
int orc_lattice(int style /*0 sc, 1 bcc, 2 fcc*/, int nx, int ny, int nz,
                double scale, double *x);
/* lattice constant for lj units from reduced density (src/lattice.cpp:249-256) */
double orc_lj_lattice_scale(int style, double rhostar);
/* velocity all create T seed [dist uniform|gaussian] [mom yes] [loop geom|all] */
int orc_velocity_create(orc_sim *s, double t_desired, int seed, int gaussian,
                        int loop_geom, int mom);

#ifdef __cplusplus
}
#endif
#endif
