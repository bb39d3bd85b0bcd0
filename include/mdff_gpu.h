/*
 * mdff_gpu.h -- C ABI of the B200 force engine for MDFF.
 *
 * The library replaces the body of the reference's per-step energy/force call
 *   SUBROUTINE engforce            (src/engforce_driver.f90:102-190)
 * which takes no arguments and communicates through module globals
 * (config.f90:47-95, coulomb.f90:47-79, pim.f90:63-96, non_bonded.f90:58-116,
 * control.f90:35-66, thermo.f90:27-120).  Here the same state crosses the
 * boundary explicitly: static force-field parameters once (mdff_gpu_create),
 * positions per call (mdff_gpu_engforce), results into caller-owned host
 * arrays.  Plain C types only; no CUDA or torch types appear in signatures.
 *
 * Array conventions
 *   - Per-type tables use 0-based C indexing [it][jt] (and [it][jt][kt]);
 *     element [it][jt] is the reference's namelist entry (it+1, jt+1).
 *     A Fortran caller transposes (see the iso_c_binding shim).
 *   - Ions are grouped by type in POSFF order: natmi[0] ions of type 0 first,
 *     then natmi[1] of type 1, ... (read_pos.f90:187-199).
 *   - Cell matrix A[a][b] = simu_cell%A(a+1,b+1): column b is lattice vector b.
 *   - Dipoles / fields: [natm][3] with xyz fastest, i.e. Fortran mu(3,natm).
 *   - 3x3 tensors: [a][b] = Fortran tau(a+1,b+1).
 *
 * Every entry point returns an int status (MDFF_OK = 0); none exits or STOPs.
 */
#ifndef MDFF_GPU_H
#define MDFF_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define MDFF_NTYPEMAX 16   /* config.f90:42 ntypemax */
#define MDFF_ASPC_DEPTH 5  /* coulomb.f90:435 dipia_ind_t(5,3,natm) */
#define MDFF_ABI_VERSION 1

/* status codes */
enum {
  MDFF_OK = 0,
  MDFF_ERR_BAD_ARGS = 1,       /* invalid argument or parameter combination   */
  MDFF_ERR_CUDA = 2,           /* CUDA runtime error (message via last_error)  */
  MDFF_ERR_CATASTROPHE = 3,    /* polarisation catastrophe, any mu_a > 10 eA
                                  (moment_from_pola.f90:176-216)               */
  MDFF_ERR_LIST_OVERFLOW = 4,  /* Verlet list capacity exceeded
                                  (tools.f90:337-350); stats.list_needed holds
                                  the required size                            */
  MDFF_ERR_NOT_CONVERGED = 5,  /* dipole solve hit its iteration limit and
                                  params.fail_on_nonconvergence is set         */
  MDFF_ERR_TIMEOUT = 6,        /* a bounded device wait gave up                */
  MDFF_ERR_NO_DEVICE = 7,      /* no CUDA device / sm_100 device unavailable   */
  MDFF_ERR_UNSUPPORTED = 8,    /* feature of the reference not built here      */
  MDFF_ERR_NOMEM = 9           /* device allocation failed                     */
};

/* control%calc (control.f90); selects the ASPC predictor use
   (moment_from_pola.f90:374-378, 415) */
enum { MDFF_CALC_MD = 0, MDFF_CALC_OPT = 1, MDFF_CALC_OTHER = 2 };

/* non_bonded ctrunc (non_bonded.f90:253-255) */
enum { MDFF_TRUNC_NONE = 0, MDFF_TRUNC_LINEAR = 1, MDFF_TRUNC_QUADRATIC = 2 };

/* &gputag keywords (new; not in the reference) */
enum { MDFF_PREC_FP64 = 0, MDFF_PREC_MIXED = 1 };
enum { MDFF_SOLVER_SCF = 0, MDFF_SOLVER_CG = 1 };
/* thole_function_type (coulomb.f90:72) */
enum { MDFF_THOLE_NONE = 0, MDFF_THOLE_LINEAR = 1, MDFF_THOLE_EXPON1 = 2, MDFF_THOLE_EXPON2 = 3,
       MDFF_THOLE_GAUSS = 4 };
/* algo_moment_from_pola (pim.f90:89-91; dispatch moment_from_pola.f90:116-127).
   KO_V3 and KO_V4_2 are rejected with MDFF_ERR_UNSUPPORTED: the reference's
   kO_v3 never forms a new dipole increment (dmu_ind stays at its zero
   initial value, moment_from_pola.f90:1716,1835) and kO_v4_2 reads
   mu_h(:,:,0) at its first iteration (:2186). */
enum { MDFF_ALGO_SCF = 0, MDFF_ALGO_KO_V1 = 1, MDFF_ALGO_KO_V2 = 2, MDFF_ALGO_KO_V3 = 3,
       MDFF_ALGO_KO_V4_1 = 4, MDFF_ALGO_KO_V4_2 = 5 };
/* algo_ext_dipole (pim.f90:85-87): predictor of the kO algorithms */
enum { MDFF_EXT_ASPC = 0, MDFF_EXT_POLY = 1 };

typedef struct mdff_params {
  int natm;                               /* config%natm                        */
  int ntype;                              /* config%ntype                       */
  int natmi[MDFF_NTYPEMAX];               /* ions per type (POSFF order)        */

  /* &controltag (control.f90:128-161) */
  int lcoulomb, lbmhft, lbmhftd, lnmlj;   /* potentials switched on             */
  int lsurf;                              /* Ewald surface term                 */
  int lreduced;                           /* reduced units: coul_unit = press_unit = 1 */
  int calc;                               /* MDFF_CALC_*                         */
  double cutshortrange, cutlongrange;     /* Angstrom                           */
  double skindiff;                        /* Verlet skin                        */

  /* &fieldtag / coulomb (coulomb.f90:55-58) */
  double qch[MDFF_NTYPEMAX];              /* charge per type                    */
  double dip[MDFF_NTYPEMAX][3];           /* static dipole per type             */

  /* &non_bondedtag (non_bonded.f90:135-150) */
  int trunc;                              /* MDFF_TRUNC_* for n-m LJ             */
  int symmetric_pot_nb;                   /* symmetrise tables (default 1)       */
  double epslj[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double sigmalj[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double plj[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double qlj[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double Abmhftd[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double Bbmhftd[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double Cbmhftd[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double Dbmhftd[MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double BDbmhftd[MDFF_NTYPEMAX][MDFF_NTYPEMAX];

  /* &coulombtag (coulomb.f90:97-106) */
  double alphaES;                         /* Ewald alpha (1/Angstrom)           */
  int kES[3];                             /* kmax per reciprocal axis           */
  int lautoES;                            /* DL_POLY rule from epsw             */
  double epsw;

  /* &pimtag (pim.f90:258-279) */
  int ldip_polar[MDFF_NTYPEMAX];
  double poldip[MDFF_NTYPEMAX][3][3];     /* polarisability tensor per type     */
  int ldip_damping[MDFF_NTYPEMAX][MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double pol_damp_b[MDFF_NTYPEMAX][MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double pol_damp_c[MDFF_NTYPEMAX][MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  int pol_damp_k[MDFF_NTYPEMAX][MDFF_NTYPEMAX][MDFF_NTYPEMAX];
  double conv_tol_ind;
  int min_scf_pol_iter, max_scf_pol_iter;
  int extrapolate_order;                  /* ASPC order 0..4                    */
  int symmetric_pot_pim;                  /* symmetrise damping tables          */

  /* &gputag (new keywords; defaults reproduce the reference) */
  int precision;                          /* MDFF_PREC_FP64 | MDFF_PREC_MIXED    */
  int solver;                             /* MDFF_SOLVER_SCF | MDFF_SOLVER_CG    */
  double cg_tol;                          /* CG stop: rms residual (e/A^2)       */
  int cg_max_iter;
  int fail_on_nonconvergence;
  int device;                             /* CUDA device ordinal                 */
  double wall24[MDFF_NTYPEMAX][MDFF_NTYPEMAX]; /* optional W/r^24 repulsive wall
                                             added to BMH pairs (eV A^24);
                                             0 = reference behaviour           */

  /* &coulombtag Thole functions (coulomb.f90:65-72, 173-175, 228-234): the
     dipole-dipole field and energy of pairs of polarisable ions use damped
     radial functions (ewald_dir.f90:305-430); forces keep the plain tensor,
     as in the reference.  thole_param[ta][tb] is used as given (ta = type of
     the pair's "ia"); mdff_b200.mdffio applies the reference's fixed values
     for expon1 / expon2 / gauss.  A = (alpha_xx(ta) alpha_xx(tb))^(1/6).     */
  int thole_type;                         /* MDFF_THOLE_*; NONE = off          */
  double thole_param[MDFF_NTYPEMAX][MDFF_NTYPEMAX];

  /* &pimtag dipole algorithm of the SCF solver (pim.f90:72, 85-91, 127-131).
     MDFF_ALGO_SCF is moment_from_pola_scf (always the ASPC predictor); the
     kO algorithms need solver = MDFF_SOLVER_SCF and alpha_xx, alpha_yy,
     alpha_zz > 0 on polarisable types; KO_V4_1 keeps at most 100 iterates
     (max_scf_pol_iter <= 100, as the reference's history arrays). */
  int algo_moment_from_pola;              /* MDFF_ALGO_*                        */
  int algo_ext_dipole;                    /* MDFF_EXT_*: kO_v1 / kO_v2 predictor */
  double omegakO;                         /* kO relaxation weight (0.7)         */

  /* &pimtag Wannier centres (pim.f90:93-96, 134-136; moment_from_pola.f90:
     136-147, 632-807).  Ions of a type with lwfc < 0 are Wannier centres;
     when some type has lwfc > 0, every other ion gets the dipole
     -2 sum (r_wfc - r_ion) over the centres with |r|^2 < rcut_wfc (the
     reference compares the squared distance with rcut_wfc itself), added
     to its total dipole after the induced-dipole solve when ldip_wfc; an
     ion of a type with lwfc > 0 must find exactly lwfc centres
     (MDFF_ERR_BAD_ARGS otherwise).  Centre types come after all other
     types, as the reference's list bookkeeping needs. */
  int lwfc[MDFF_NTYPEMAX];
  int ldip_wfc;                           /* default 1                          */
  double rcut_wfc;                        /* default 0.5                        */
} mdff_params;

/* Results of one engforce call; pointer members are caller-owned host arrays
   (NULL = not wanted, except fx/fy/fz). */
typedef struct mdff_result {
  double *fx, *fy, *fz;                   /* [natm] forces (eV/A)                */
  double *mu;                             /* [natm][3] total dipoles mu_t        */
  double *ef;                             /* [natm][3] field ef_t (e/A^2)        */
  double u_lj, vir_lj;                    /* thermodynamic module scalars        */
  double u_bmhft, vir_bmhft;
  double u_coul, u_pol, pvirial_coul;
  double tau_nonb[3][3];                  /* GPa                                 */
  double tau_coul[3][3];
  double tau[3][3];                       /* tau_nonb + 2 tau_coul, as the
                                             reference's double accumulation
                                             (ewald.f90:245 + engforce_driver.f90:177) */
} mdff_result;

typedef struct mdff_stats {
  int n_pol_iter;                         /* SCF or CG iterations last call      */
  int converged;
  double rmsd;                            /* final rmsd (e/A^2)                  */
  int list_rebuilds;                      /* cumulative                          */
  int list_capacity;                      /* full-list entries allocated         */
  int list_needed;                        /* entries needed at last build        */
  int nk;                                 /* half-space k vectors                */
  double alphaES;                         /* after lautoES                       */
  int kES[3];
  double cutlongrange;                    /* after the half-cell clamp           */
  int n_launches;                         /* kernels launched by last call       */
  double ms_last;                         /* device time of last call (ms)       */
  double rmsd_initial;                    /* CG: rmsd of the first guess (e/A^2) */
  int n_fp64_residuals;                   /* CG: FP64 residual evaluations       */
  int n_kardir;                           /* in-place kardir/dirkar round trips
                                             the reference's engforce makes for
                                             this call (one per short-range
                                             routine, per multipole_ES_dir and
                                             for the Wannier centres); -1 when
                                             the solve is not the reference's
                                             SCF.  The MD loop's vnlistcheck
                                             (runmd.f90:304) adds one more, three
                                             when it rebuilds (tools.f90:474-526) */
} mdff_stats;

typedef struct mdff_ctx* mdff_handle;

int mdff_gpu_abi_version(void);
/* sizeof the boundary structs as compiled into the library: which = 0
   mdff_params, 1 mdff_result, 2 mdff_stats (bindings check their layout) */
int mdff_gpu_struct_size(int which);
const char* mdff_gpu_strerror(int status);
/* last CUDA / validation message of this handle (or global if h == NULL) */
const char* mdff_gpu_last_error(mdff_handle h);

/* Replaces field_init / coulomb_init / pim_init / initialize_param_non_bonded
   (non_bonded.f90:455-644, coulomb.f90:363-493, pim.f90:107-240,
   read_pos.f90:160-237): expands per-type tables to ions, symmetrises,
   clamps cutlongrange to half the cell (coulomb.f90:377-383), applies lautoES,
   builds the k mesh (kspace.f90:143-207).  cell_A as in simu_cell%A. */
int mdff_gpu_create(const mdff_params* p, const double cell_A[9], mdff_handle* out);

/* New cell (lattice.f90:60): rebuilds B, omega, k mesh; forces a list rebuild. */
int mdff_gpu_set_cell(mdff_handle h, const double cell_A[9]);

/* engforce (engforce_driver.f90:102-190) on host arrays rx,ry,rz [natm].
   itime drives the ASPC order ramp (moment_from_pola.f90:514-522).  The
   Verlet list is checked (tools.f90:444-537) and rebuilt on device as needed. */
int mdff_gpu_engforce(mdff_handle h, const double* rx, const double* ry,
                      const double* rz, int itime, mdff_result* out);

/* Same on device-resident arrays: d_pos = SoA [3][natm] doubles; outputs are
   device arrays d_force [3][natm] (required), d_mu / d_ef [natm][3]
   (optional); scalars/tensors go to *out (its pointer members are ignored).
   The call is stream-ordered on the handle's stream and returns after the
   scalars are on the host. */
int mdff_gpu_engforce_device(mdff_handle h, const double* d_pos, int itime,
                             double* d_force, double* d_mu, double* d_ef,
                             mdff_result* out);

/* The reference converts the global positions to direct coordinates and
   back in place around each pass over the pairs (kardir / dirkar,
   lattice.f90:183-270; ewald_dir.f90:138,739, non_bonded.f90:1113,1221,
   moment_from_pola.f90:685,803, tools.f90:474,502), which moves them by an
   ulp or so each time; the engine leaves the caller's positions alone.  A
   caller that wants the reference's positions after an engforce applies
   count = stats.n_kardir round trips here (same cell as the handle; host
   arrays rx, ry, rz [natm], in place, in the reference's arithmetic);
   0 <= count <= 1048576, else MDFF_ERR_BAD_ARGS. */
int mdff_gpu_kardir_roundtrips(mdff_handle h, double* rx, double* ry, double* rz, int count);

/* ASPC history dipia_ind_t(5,3,natm) (coulomb.f90:435) for RESTART:
   buf = [MDFF_ASPC_DEPTH][natm][3]. */
int mdff_gpu_get_aspc_history(mdff_handle h, double* buf);
int mdff_gpu_set_aspc_history(mdff_handle h, const double* buf);

int mdff_gpu_get_stats(mdff_handle h, mdff_stats* s);

/* Export the reference's half Verlet list (vnlist_pbc, tools.f90:273-368) for
   positions rx,ry,rz: which = 0 -> verlet_vdw (cutshortrange + skindiff),
   1 -> verlet_coul (cutlongrange + skindiff).  point[natm+1] and list[] are
   1-based exactly as the reference (list order ascending ja within a row).
   *n_out = number of entries; MDFF_ERR_LIST_OVERFLOW if capacity is short. */
int mdff_gpu_verlet_half_list(mdff_handle h, int which, const double* rx,
                              const double* ry, const double* rz, int* point,
                              int* list, int capacity, int* n_out);

/* The same half list as mdff_gpu_verlet_half_list, computed without any
   device allocation and without a handle: all scratch lives in one
   file-scope static device array of about 18.4 MB that every GPU loading the
   library holds until exit.  It has no counterpart in the reference.  It is
   for callers that cannot call cudaMalloc, e.g. a host program whose device
   memory is owned by another runtime's caching pool (where a cudaMalloc can
   fail or fragment that pool), or a utility that needs only the list and
   should not create an engine.  Host inputs / outputs as for
   mdff_gpu_verlet_half_list; params supplies natm, the cutoffs, skindiff,
   lcoulomb (half-cell clamp of cutlongrange) and device.  Limits of the
   static array: natm <= 32768, list entries <= 4194304 and at most 4096
   entries in one row; beyond any of them the call returns MDFF_ERR_BAD_ARGS
   with a message on stderr (*n_out holds the entry count when the entry
   limit was the one exceeded).  MDFF_ERR_LIST_OVERFLOW means only that
   capacity is below *n_out: grow list and call again.  The first call on a
   device looks up the array's address.  Every call shares the one array and
   clears what it needs: two calls overlapping on the same GPU (from two
   host threads) race on it. */
int mdff_gpu_verlet_half_list_noalloc(const mdff_params* p, const double cell_A[9], int which,
                                      const double* rx, const double* ry, const double* rz,
                                      int* point, int* list, int capacity, int* n_out);

/* Velocity-Verlet NVE steps on device (prop_velocity_verlet,
   integration.f90:132-194): d_pos, d_vel SoA [3][natm], d_invmass [natm] in
   internal units, dt in internal time units.  Each step calls the engine.
   ekin_pot (optional host [nsteps][2]) receives kinetic and potential energy
   per step (eV). */
int mdff_gpu_md_nve(mdff_handle h, double* d_pos, double* d_vel,
                    const double* d_invmass, double dt, int nsteps, int itime0,
                    double* ekin_pot);

/* Electric field gradient efg_t (doefg; ewald_dir.f90:543-582,
   ewald_rec.f90:209-217, ewald.f90 self term) at every ion for the state of
   the last engforce call (its positions and total dipoles): efg [natm][3][3]
   host array, eV/(e A^2) (x coul_unit as the reference).  The reciprocal part
   fills the upper triangle only, as the reference does.  FP64. */
int mdff_gpu_efg(mdff_handle h, double* efg);

/* Per-kernel-class device timing with CUDA events on the handle's stream
   (for roofline figures).  Classes: 0 list build, 1 short range, 2 real-space
   field, 3 real-space force, 4 structure factor, 5 reciprocal field/force,
   6 everything else.  ms[c], launches[c] and work[c] accumulate while enabled
   (reset on enable); work is the algorithmic op count of the reciprocal
   classes 4 and 5 ((k, ion) terms x ops per term), 0 for the others. */
#define MDFF_NKCLASS 7
int mdff_gpu_profile(mdff_handle h, int enable);
int mdff_gpu_kernel_times(mdff_handle h, double* ms, long long* launches, double* work);

/* Test hook for the timeout path; no counterpart in the reference.  polls =
   how many times the tensor-core structure factor of the mixed engine's CG
   operator polls, before it gives up, the mbarrier that frees an operand
   stage (each poll may suspend the thread for up to 1 us); polls < 0 restores
   the default of 2^22.  With polls = 0 every such wait gives up at once: the
   kernel stops issuing matrix products, waits with the default bound for the
   products already issued, frees its tensor memory and returns, and the
   engforce call returns MDFF_ERR_TIMEOUT.  The setting stays on the handle
   until changed; the handle remains usable. */
int mdff_gpu_set_tc_wait_limit(mdff_handle h, int polls);

/* Measured FMA throughput of a device (TFLOP/s, FMA = 2 flops) for fp64 = 1
   (double) or 0 (float): a saturating register-resident FMA loop over every
   SM, timed with CUDA events.  The denominator of the FP32/FP64 roofline. */
int mdff_gpu_peak_flops(int device, int fp64, double* tflops);

void mdff_gpu_destroy(mdff_handle h);

/* ---- batched evaluation ------------------------------------------------------
   No counterpart in the reference, which evaluates one configuration per
   engforce call.  Many independent configurations (each its own cell, ion
   count and composition; up to MDFF_BATCH_MAXTYPES types and
   MDFF_BATCH_MAXATM ions) are evaluated by one persistent kernel launched
   through a CUDA graph: one thread-block cluster per configuration, taken from
   a device queue in descending cost order.  Each configuration is one
   engforce (engforce_driver.f90:102-190) with calc = 'other' (no ASPC
   history): forces, energies, stress, dipoles and fields, the dipoles from PCG
   (cg_tol, else conv_tol_ind; cg_max_iter).  precision of parameter set 0
   selects FP64 or mixed for the whole batch.  The real-space pairs are all
   minimum-image pairs within the cutoffs (the Verlet list's pair set).
   Thole functions and Wannier centres act as in mdff_gpu_create (a missing
   centre: MDFF_ERR_BAD_ARGS).  The dipoles always come from PCG: a parameter
   set that selects kO_v1, kO_v2 or kO_v4_1 gets that algorithm's converged
   dipoles (its fixed point, to the tolerance), not its iteration path or
   iteration count, which mdff_gpu_create reproduces. */
#define MDFF_BATCH_MAXTYPES 4
#define MDFF_BATCH_MAXATM 2048

typedef struct mdff_batch* mdff_batch_handle;

typedef struct mdff_batch_desc {
  int nconf;
  const int* pset;            /* [nconf] parameter set of each configuration       */
  const int* natmi;           /* [nconf][MDFF_NTYPEMAX] ions per type (grouped)     */
  const double* cell_A;       /* [nconf][9] simu_cell%A, row-major as in create     */
} mdff_batch_desc;

/* per-configuration outputs (the mdff_result scalars plus solver and set-up
   figures) */
typedef struct mdff_batch_conf {
  double u_lj, vir_lj, u_bmhft, vir_bmhft, u_coul, u_pol, pvirial_coul;
  double tau_nonb[3][3], tau_coul[3][3], tau[3][3];
  double rmsd;                /* final dipole residual (e/A^2)                      */
  int n_pol_iter, converged, catastrophe, nk;
  double alphaES, cutlongrange;
  int kES[3], pad;
} mdff_batch_conf;

/* psets[npsets]: parameter sets (natm / natmi of a set are ignored: each
   configuration takes them from desc).  Positions of configuration c occupy
   entries off_c .. off_c + natm_c - 1 of the concatenated arrays, off_c =
   sum of the earlier configurations' ion counts. */
int mdff_gpu_batch_create(const mdff_params* psets, int npsets, const mdff_batch_desc* desc,
                          mdff_batch_handle* out);
/* host arrays rx, ry, rz [ntot]; fx, fy, fz [ntot] (required); mu, ef
   [ntot][3] (optional); conf [nconf] (optional) */
int mdff_gpu_batch_engforce(mdff_batch_handle h, const double* rx, const double* ry,
                            const double* rz, double* fx, double* fy, double* fz, double* mu,
                            double* ef, mdff_batch_conf* conf);
/* device arrays: d_pos, d_force SoA [3][ntot]; d_mu, d_ef [ntot][3] (optional);
   conf (host, optional) */
int mdff_gpu_batch_engforce_device(mdff_batch_handle h, const double* d_pos, double* d_force,
                                   double* d_mu, double* d_ef, mdff_batch_conf* conf);
/* Autotuner: times every launch shape (cluster size x threads per CTA) on the
   positions of the last call and keeps the fastest; returns it and its time. */
int mdff_gpu_batch_tune(mdff_batch_handle h, int* cluster, int* threads, double* ms);
/* force a launch shape (cluster 1, 2, 4 or 8; threads 256 or 512) */
int mdff_gpu_batch_set_shape(mdff_batch_handle h, int cluster, int threads);
/* ntot, nconf, the launch shape and the device time of the last call */
int mdff_gpu_batch_info(mdff_batch_handle h, int* ntot, int* nconf, int* cluster, int* threads,
                        double* ms_last);
const char* mdff_gpu_batch_last_error(mdff_batch_handle h);
void mdff_gpu_batch_destroy(mdff_batch_handle h);

/* ---- force-field gradients of a batch (differentiable fitting) -------------
   No counterpart in the reference.  Fit parameters (at most MDFF_FIT_MAX),
   each a kind and type indices, act on every parameter set of the batch:
     MDFF_FIT_A / _RHO / _C   Buckingham A (eV), rho (A, B = 1/rho), C (eV A^6)
                              of the type pair (t1, t2), both orders
     MDFF_FIT_POL             isotropic polarisability of type t1 (A^3)
     MDFF_FIT_TTB / _TTC      Tang-Toennies b (1/A), c of the charge field of
                              type t2 on the dipoles of type t1: pol_damp
                              (t1,t1,t2) and (t1,t2,t1)
     MDFF_FIT_QSCALE          one factor s on every charge (qch * s)
   mdff_gpu_batch_adjoint returns dJ/dtheta for J = sum_c [ gE_c U_c + gF . F
   + gmu . mu_ind ] (U = u_lj + u_bmhft + u_coul, eV) at the positions of the
   last evaluation: one adjoint linear solve per configuration with the
   dipole solver's operator.  gE [nconf], gF SoA [3][ntot], gmu [ntot][3] or
   NULL; host arrays (on_device = 0) or device arrays (1); grad [nparam] and
   grad_conf [nconf][nparam] (optional) are host arrays.  The surface term
   (lsurf) is not covered.  The call reuses the evaluation's device state and
   overwrites its field buffer: fetch ef before calling it. */
#define MDFF_FIT_MAX 16
#define MDFF_FIT_A 0
#define MDFF_FIT_RHO 1
#define MDFF_FIT_C 2
#define MDFF_FIT_POL 3
#define MDFF_FIT_TTB 4
#define MDFF_FIT_TTC 5
#define MDFF_FIT_QSCALE 6
int mdff_gpu_batch_fit_define(mdff_batch_handle h, int nparam, const int* kind, const int* t1,
                              const int* t2);
/* set the fit parameters' values (rebuilds every configuration's tables) */
int mdff_gpu_batch_fit_set(mdff_batch_handle h, const double* theta);
int mdff_gpu_batch_fit_get(mdff_batch_handle h, double* theta);
int mdff_gpu_batch_adjoint(mdff_batch_handle h, const double* gE, const double* gF,
                           const double* gmu, int on_device, double* grad, double* grad_conf);

#ifdef __cplusplus
}
#endif
#endif /* MDFF_GPU_H */
