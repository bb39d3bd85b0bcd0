/*
 * mdff_oracle.h -- CPU FP64 restatement of the MDFF engforce path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA engine is compared
 * against; the product (libmdff_gpu.so, mdff_b200/) never links, loads or
 * calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg use it.
 *
 * Each function restates the reference Fortran routine cited beside it, with
 * the same loop structure, inclusion tests and operation order (compiled with
 * -ffp-contract=off so no FMA contraction changes roundings).  It shares the
 * boundary types (mdff_params / mdff_result) of include/mdff_gpu.h.
 */
#ifndef MDFF_ORACLE_H
#define MDFF_ORACLE_H

#include "../include/mdff_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_ctx or_ctx;

typedef struct or_extra {
  double* efg;        /* [natm][3][3] electric field gradient (optional)    */
  int do_efg;         /* compute efg (doefg)                                 */
  int n_scf;          /* out: SCF iterations                                 */
  double rmsd;        /* out: final SCF rmsd                                 */
  double u_dir, u_rec, u_self, u_surf; /* out: parts of the final u_coul (internal units) */
  int n_kardir;       /* out: in-place kardir/dirkar round trips of the call  */
} or_extra;

or_ctx* or_create(const mdff_params* p, const double cell_A[9], int* status);
void or_destroy(or_ctx* c);
void or_set_threads(int n);
int or_get_threads(void);

/* engforce (engforce_driver.f90:102-190).  ex may be NULL. */
int or_engforce(or_ctx* c, const double* rx, const double* ry, const double* rz,
                int itime, mdff_result* out, or_extra* ex);

/* count in-place kardir/dirkar round trips (lattice.f90:183-270) of the
   positions with the context's cell */
void or_kardir_roundtrips(or_ctx* c, double* rx, double* ry, double* rz, int count);

/* vnlist_pbc (tools.f90:273-368): which = 0 vdw, 1 coul; 1-based CSR. */
int or_vnlist(or_ctx* c, const double* rx, const double* ry, const double* rz,
              int which, int* point, int* list, int capacity, int* n_out);

/* vnlistcheck (tools.f90:444-537): *disp = largest + second largest
   displacement since the last rebuild (stored direct coordinates start at
   zero, so the first call rebuilds); *rebuilt = 1 when the sum is above
   skindiff, and the positions become the new reference. */
int or_vnlistcheck(or_ctx* c, const double* rx, const double* ry, const double* rz, double* disp,
                   int* rebuilt);

int or_get_aspc(or_ctx* c, double* buf);
int or_set_aspc(or_ctx* c, const double* buf);

/* derived set-up values, for host-logic tests */
typedef struct or_setup_info {
  double alphaES; int kES[3]; int nk; double cutlongrange;
  double B[9]; double omega; double WA, WB, WC;
  int task[6];
} or_setup_info;
int or_get_setup(or_ctx* c, or_setup_info* info);
/* sorted k mesh: kx,ky,kz,kk,Ak,kcoe each [nk] (kspace.f90:143-207) */
int or_get_kmesh(or_ctx* c, double* kx, double* ky, double* kz, double* kk,
                 double* Ak, double* kcoe);

/* NR erfc (functions.f90:28-40) and TT damping (tt_damp.f90:68-97) */
double or_errfc(double x);
void or_tt_damp(double b, double c, double r, int order, double* f, double* fd);
/* polint (moment_from_pola.f90:2365-2412) at x = 1 through (xa_i, ya_i), n <= 10 */
double or_polint(const int* xa, const double* ya, int n);

#ifdef __cplusplus
}
#endif
#endif
