/*
 * desalm.h -- C ABI of the B200 pseudo-time iteration (RHS residual, diagonal
 * approximate-factorisation smoother, FAS multigrid V-cycle, Spalart-Allmaras
 * sub-iterations) of the DES-ALM artificial-compressibility solver.
 *
 * Every entry point replaces one subroutine of the reference's mg_driver call
 * chain (src/mg_driver.F90).  The reference passes Fortran explicit-shape
 * arrays q(1:me, il:iu, jl:ju, kl:ku) (component fastest, then i, j, k); the
 * host arrays of this ABI use exactly that layout, so a Fortran caller passes
 * its own arrays through ISO_C_BINDING without a copy.  On the device the
 * library keeps one structure-of-arrays block per multigrid level.
 *
 * All functions return 0 on success or a negative DESALM_E* status.  Calls on
 * one context are ordered on the context's CUDA stream and are not thread safe;
 * independent contexts are.  desalm_last_error() returns a message for the last
 * failure on a context.
 *
 * The same symbols with the prefix desalm_oracle_ are exported by the CPU
 * restatement used as the test oracle (oracle/); it is not part of the product.
 */
#ifndef DESALM_H
#define DESALM_H

#ifdef __cplusplus
extern "C" {
#endif

#define DESALM_ABI_VERSION 1

/* status codes */
#define DESALM_OK          0
#define DESALM_EINVAL     -1   /* bad argument or unsupported case setting      */
#define DESALM_ENOMEM     -2   /* device or host allocation failed              */
#define DESALM_ECUDA      -3   /* CUDA runtime error                            */
#define DESALM_ENONFINITE -4   /* NaN/Inf in the convergence norm               */
#define DESALM_ESINGULAR  -5   /* zero pivot in a line solve                    */
#define DESALM_ETIMEOUT   -6   /* bounded device wait gave up                   */
#define DESALM_ENOTREADY  -7   /* grid or state not bound yet                   */
#define DESALM_EIO        -8   /* file missing, unreadable, or not in the
                                  expected record layout                        */

/* precision_mode */
#define DESALM_FP64   0        /* everything in FP64                            */
#define DESALM_MIXED  1        /* FP64 state, residual, restriction, update
                                  and norm on every level; FP32 DAF line
                                  sweeps, modal transforms, prolongation
                                  correction and turbulence ADI              */
/* predictor: initial guess of q^{n+1} for the pseudo-time loop */
#define DESALM_PRED_QN      0  /* q^n, as src/mg_driver.F90:50-51              */
#define DESALM_PRED_LINEAR  1  /* 2 q^n - q^{n-1}                               */
#define DESALM_PRED_LEARNED 2  /* 2 q^n - q^{n-1} + a correction from a 3D conv
                                  network trained online on the solver's own
                                  time levels (desalm_lp_* below)               */

/* boundary types, as documented at the end of ind3dmg.dat (nbtype) */
#define DESALM_BC_INTERFACE 0
#define DESALM_BC_WALL      1
#define DESALM_BC_SYMMETRY  2
#define DESALM_BC_FREESTREAM 3
#define DESALM_BC_INFLOW    4
#define DESALM_BC_OUTLET    5   /* characteristics (LODI) exit; solved on the i = im face */
#define DESALM_BC_PERIODIC  6

/* Case description: the part of ind3dmg.dat (read in src/init.F90:176-236)
 * and of the compile-time switches (src/global.F90, src/global_param.F90)
 * that the pseudo-time iteration uses.  Sizes are node counts including the
 * boundary nodes (one block, one rank: no ghost layers). */
typedef struct desalm_case {
    int    im, jm, km;      /* fine-grid nodes: img(1), jmg(1), kmg(1)         */
    int    ng;              /* multigrid levels, 1..4 (ng in src/global.F90)    */
    int    icrs, jcrs, kcrs;/* 1 = full coarsening in that direction, 0 = none  */
    int    iter[4];         /* smoothing iterations per level: iter(n)          */
    int    itmax;           /* itm(1): pseudo-iterations per physical step      */
    int    it_min;          /* minimum pseudo-iterations before convergence     */
    double er_min, eo_min;  /* log10 drop / absolute tolerances                 */
    double delti;           /* physical time step                               */
    double ren, beta;       /* Reynolds number, artificial compressibility      */
    double cfl1, vnn1;      /* local pseudo-time step limits (mean flow)        */
    double cfl2, vnn2;      /* local pseudo-time step limits (turbulence)       */
    int    itk;             /* SA sub-iterations per call                       */
    double ep[2][3];        /* ep(1,:) DAF implicit smoothing, ep(2,:) prolongation smoothing */
    double pdiss_coef;      /* pressure dissipation coefficient                 */
    int    btype[6], bdir[6];
    int    ifix, jfix, kfix;/* 1-based pressure reference node                  */
    int    turbulence;      /* 0: laminar (nu_t = 0); 1: Spalart-Allmaras;
                               2: Wilcox k-omega (k in q(5), omega through
                               desalm_set_omega)                              */
    int    unsteady;        /* e_source = 1 (BDF2 physical time terms) or 0     */
    int    conservation;    /* 1: outlet mass-flux fix once per physical step   */
    int    precision_mode;  /* DESALM_FP64 or DESALM_MIXED                      */
    int    predictor;       /* DESALM_PRED_*                                    */
    int    use_graph;       /* 1: replay each pseudo-iteration as a CUDA graph  */
    int    wall_functions;  /* 1: wf_eta(1) and wf_eta(2) after every fine DAF
                               step (src/mg_driver.F90:221-224); 0 (the
                               default): off, as for wall-resolved grids     */
    int    reserved[5];
} desalm_case;

/* Outcome of one physical time step (desalm_mg_driver). */
typedef struct desalm_step_report {
    int    iterations;      /* pseudo-iterations taken (itc)                    */
    int    converged;       /* 1 if the mg_ck_conver test passed                */
    double residual[5];     /* last log10 mean |q - q_old| per field            */
    double init_residual[5];/* first-iteration values (init_resd)               */
    int    pivots;          /* rows interchanged by partial pivoting in the line
                               solves (SGTSV, src/sgtsv.f:107-135): a line
                               system with a column that is not diagonally
                               dominant is solved by the pivoting elimination;
                               the others need no interchange               */
    int    pivot_lines;     /* line systems that took the pivoting elimination
                               (a column not diagonally dominant), summed over
                               the step's sweeps; the others were solved by
                               the no-interchange elimination               */
    int    reserved[6];
} desalm_step_report;

/* fields for desalm_get_field / desalm_set_field (SoA, one level) */
enum desalm_field {
    DESALM_F_Q = 0,        /* +m, m = 0..4 (p, u, v, w, nu_tilde)               */
    DESALM_F_QN = 8,       /* +m                                               */
    DESALM_F_QNM1 = 16,    /* +m                                               */
    DESALM_F_QOLD = 24,    /* +m  (qold_mg)                                    */
    DESALM_F_RH = 32,      /* +m, m = 0..3                                     */
    DESALM_F_PK = 40,      /* +m, m = 0..3                                     */
    DESALM_F_CSI = 48,     /* +d, d = 0..2                                     */
    DESALM_F_ETA = 52,
    DESALM_F_ZET = 56,
    DESALM_F_AJ = 60,
    DESALM_F_NUT = 61,
    DESALM_F_DTAU = 62,
    DESALM_F_DTEV = 63,
    DESALM_F_WD = 64,
    DESALM_F_X = 65, DESALM_F_Y = 66, DESALM_F_Z = 67
};

typedef struct desalm_ctx desalm_ctx;

/* Context life cycle.  Replaces init_mg / init_daf_bc (src/init.F90:1025,439):
 * validates the case and allocates every level's device arrays once. */
int  desalm_init(const desalm_case* c, desalm_ctx** out);
void desalm_destroy(desalm_ctx* ctx);
const char* desalm_last_error(const desalm_ctx* ctx);
/* Level extents (1-based level n): writes im, jm, km. */
int  desalm_level_dims(const desalm_ctx* ctx, int n, int dims[3]);

/* Fine-grid coordinates x(i,j,k), y, z (i fastest) and the wall distance
 * (nullable; needed for SA).  Injects the grid to the coarse levels
 * (src/mg_inject.F90:26-62), computes metrics and Jacobians on every level
 * (src/mg_metrics.F90:56-250), the SA pseudo-time step dtev
 * (src/mg_metrics.F90:262-282) and the inflow extrapolation ratios rat
 * (src/init.F90:2750-2891). */
int  desalm_set_grid(desalm_ctx* ctx, const double* x, const double* y,
                     const double* z, const double* wd);

/* Fine-level state in the reference's layout q(1:5, i, j, k) (src/global.F90:62);
 * nut is xnut(i,j,k).  qn/qnm1/nut may be NULL (then zero).  Replaces the
 * 'solu' reader (src/init.F90:2392-2411). */
int  desalm_set_state(desalm_ctx* ctx, const double* q, const double* qn,
                      const double* qnm1, const double* nut);
int  desalm_get_state(desalm_ctx* ctx, double* q, double* qn, double* qnm1,
                      double* nut);

/* The same three calls for FP32 host arrays in the same layouts: the
 * reference's q, qn, qnm1, xnut, x, y, z and wd are real(rdf) = FP32
 * (src/precision.F90:11), so a Fortran caller passes them without keeping a
 * double copy.  Values are widened to FP64 on the way in and rounded to
 * nearest on the way out. */
int  desalm_set_state_f32(desalm_ctx* ctx, const float* q, const float* qn,
                          const float* qnm1, const float* nut);
int  desalm_get_state_f32(desalm_ctx* ctx, float* q, float* qn, float* qnm1,
                          float* nut);
int  desalm_set_grid_f32(desalm_ctx* ctx, const float* x, const float* y,
                         const float* z, const float* wd);

/* One SoA field of one level (values converted to/from double). */
int  desalm_get_field(desalm_ctx* ctx, int n, int field, double* out);
int  desalm_set_field(desalm_ctx* ctx, int n, int field, const double* in);

/* One DAF smoother step on level n: src/solver_daf.F90:2-488
 * (solver_daf(me, n, decide_recalc_rh, itr, ...)). */
int  desalm_solver_daf(desalm_ctx* ctx, int n, int recalc, int itr);
/* FAS restriction + injection to level n, then mg_zero_pk_boundary:
 * src/mg_nlevel.F90:2-146 and src/mg_driver.F90:134,407-466. */
int  desalm_mg_nlevel(desalm_ctx* ctx, int n);
/* Coarse-grid correction from level n+1 to level n: src/mg_prolong.F90:2-277
 * with src/rsmooth.F90:7-95 and src/rs_sweep.F90:111-291. */
int  desalm_mg_prolong(desalm_ctx* ctx, int n);
/* log10 of mean |q - qold_mg| per field over interior nodes of level n:
 * src/mg_residual.F90:2-84. */
int  desalm_mg_residual(desalm_ctx* ctx, int n, double res[5]);
/* Fine-grid boundary conditions and pressure fix: src/bcond_fm.F90:2-322. */
int  desalm_bcond_fm(desalm_ctx* ctx);
/* Spalart-Allmaras sub-iterations on the fine level: src/des_eddy.F90:2-297. */
int  desalm_des_eddy(desalm_ctx* ctx);
/* k-omega sub-iterations on the fine level (turbulence = 2): kw_eddy,
 * src/kw_eddy.F90:2-296, with rhs_kw_ptke, rhs_kw_coef, rhs_kw_prod,
 * rhs_kw_viscous, rhs_kw_flux, rhs_kw_unst_visc, rhs_kw_implicit_source and
 * rhs_kw_bcond.  k is q(5); omega is the reference's q(6), set and read
 * with desalm_set_omega / desalm_get_omega as (i, j, k) arrays of its three
 * time levels.  desalm_mg_driver and desalm_pseudo_iteration call it where
 * the reference's driver calls des_eddy.  The reference does not build this
 * model (kw_eddy.F90 is not in its makefile and its ADI file
 * rhs_kw_adi_solver_ijk.F90 does not exist): the ADI here follows the SA
 * model's (src/rhs_sa_adi_solver.F90:50-244) for each of k and omega.
 * nu_t = As k / omega on every node after each sub-iteration, as
 * rhs_kw_bcond sets it (src/rhs_kw_bcond.F90:477-491).  A case with wall
 * faces needs the wall distance given to desalm_set_grid. */
int  desalm_kw_eddy(desalm_ctx* ctx);
/* omega (q(6)), its previous time level qn(2) and the one before qnm1(2)
 * of the fine level, (i, j, k) with i fastest; omega_n / omega_nm1 may be
 * NULL (zero on set, skipped on get). */
int  desalm_set_omega(desalm_ctx* ctx, const double* omega, const double* omega_n,
                      const double* omega_nm1);
int  desalm_get_omega(desalm_ctx* ctx, double* omega, double* omega_n, double* omega_nm1);
/* Floors of k and omega on extrapolated, outlet and periodic faces: ckin,
 * cein of ind3dmg.dat (read at src/init.F90:188, applied in
 * src/rhs_kw_bcond.F90).  Defaults 1e-10 and 1e-6. */
int  desalm_kw_config(desalm_ctx* ctx, double ckin, double cein);
/* Outlet mass-flux correction: src/conservation.F90:2-162. */
int  desalm_conservation(desalm_ctx* ctx);
/* Log-law wall functions on the fine level's j walls, wf_eta(1) and
 * wf_eta(2) (src/wf_mpi.F90:246-413), which the reference's mg_driver calls
 * after every fine solver_daf (src/mg_driver.F90:221-224);
 * desalm_mg_driver / desalm_pseudo_iteration do the same when
 * desalm_case.wall_functions = 1.  Layer 2 (j = 2 and jm-1) gets the wall
 * law's speed at its wall distance in the direction of layer 3's
 * wall-parallel velocity, and nu_tilde = kappa y+ / Re; u_tau solves the
 * reference's wall law (funcv, src/wf_mpi.F90:602-628) to full precision,
 * where the reference stops its Newton search at |F| < 1e-4.  Needs the
 * wall distance given to desalm_set_grid. */
int  desalm_wall_functions(desalm_ctx* ctx);
/* qold_mg <- q on the fine level (src/mg_driver.F90:98-100). */
int  desalm_save_qold(desalm_ctx* ctx);
/* Start of a physical time step (src/mg_driver.F90:42-75): qnm1 <- qn,
 * qn <- q, the predictor's initial guess, injection of qn/qnm1 to the coarse
 * levels, the optional mass-flux fix, and qold_mg <- q. */
int  desalm_begin_step(desalm_ctx* ctx);
/* One physical time step: src/mg_driver.F90:2-323 (history shift, coarse
 * injection of qn/qnm1, predictor, optional conservation, pseudo-time loop
 * with down-leg V-cycle, prolongation, bcond_fm and mg_ck_conver). */
int  desalm_mg_driver(desalm_ctx* ctx, desalm_step_report* rep);
/* One physical step of each of n independent blocks (contexts), as
 * desalm_mg_driver on each: the reference gives each zone its own MPI ranks
 * (myzone, src/init.F90:579-590), and each runs mg_driver on its blocks.
 * Contexts on the graph path
 * (use_graph = 1, not the learned guess) have their captured steps in
 * flight on their own streams at once, so small blocks share the GPU; the
 * others step in turn.  Each block's result equals its desalm_mg_driver
 * bit for bit (there is no exchange between blocks).  reps (n entries) may
 * be NULL.  Returns the first error; the steps already in flight are
 * finished first. */
int  desalm_mg_driver_batch(desalm_ctx* const* ctxs, int n, desalm_step_report* reps);
/* Overset blocks (the reference's zones of one grid, src/init.F90:1950-2060):
 * donee nodes of each block take the fields of a host cell in another block
 * by trilinear interpolation, mg_bintp_mom (q(1:4), src/mg_bintp_mom.F90:
 * 100-122) after every fine-level DAF step and mg_bintp_tur (the turbulence
 * fields: nu_tilde, or k and omega) after every fine-level turbulence update
 * (src/mg_driver.F90:164-183,237-244).  Entry e of the map: donee[4 e] =
 * block (index into ctxs), i, j, k (1-based) of the node that receives;
 * host[4 e] = block, i, j, k of the lower corner of the host cell, whose
 * eight corners are interpolated with the weights (1 - x or x)(1 - y or
 * y)(1 - z or z), coef[3 e] = x, y, z (xco, yco, zco).  All values are read
 * before any is written, as the reference gathers them before its
 * mpi_alltoallv.  A face whose nodes receive donor data is btype 0
 * (interface): bcond_fm leaves it alone. */
typedef struct desalm_overset_map {
  int n;
  const int* donee;
  const int* host;
  const double* coef;
} desalm_overset_map;
typedef struct desalm_overset desalm_overset;
/* The blocks (contexts on the current GPU, with the same ng, iter, itmax,
 * convergence settings, turbulence model and wall-function switch; their
 * grids and states set) and their donor map; the map is copied. */
int  desalm_overset_create(desalm_ctx* const* ctxs, int nblocks, const desalm_overset_map* map,
                           desalm_overset** out);
void desalm_overset_destroy(desalm_overset* ov);
const char* desalm_overset_last_error(const desalm_overset* ov);
/* One exchange now: what = 0 the momentum fields q(1:4), 1 the turbulence
 * fields. */
int  desalm_overset_exchange(desalm_overset* ov, int what);
/* One physical step of every block in lockstep, as the reference's
 * mg_driver runs its zones (src/mg_driver.F90:2-323): each block's begin_step,
 * then pseudo-iterations whose fine-level smoothing steps exchange donor
 * data as above; each block's kernels run on its own stream, concurrently
 * with the other blocks' between exchanges.  The convergence test
 * (mg_ck_conver) uses the sum of |q - qold_mg| over every block's interior
 * divided by the interior node count of block 0 (the reference sums over
 * all ranks and divides by its root's zone's count, src/mg_residual.F90:
 * 31,64-80).  reps (nblocks entries, may be NULL) all get the combined
 * report.  Blocks step eagerly (no CUDA graph). */
int  desalm_overset_mg_driver(desalm_overset* ov, desalm_step_report* reps);

/* Overset blocks sharded across processes (one GPU each): a rank steps the
 * blocks it owns and exchanges donor values with the other ranks, as the
 * reference fills a send buffer per destination, calls mpi_alltoallv and
 * writes what it receives (src/mg_bintp_mom.F90:60-160,
 * src/mg_bintp_tur.F90).  A list is n points on blocks of this process:
 * pts[4 p + 0] the block (index into ctxs), pts[4 p + 1..3] its 1-based
 * i, j, k.  With weights (coef[3 p + 0..2] = xco, yco, zco) the points are
 * host cells (lower corners) and desalm_ov_list_gather writes the
 * trilinear interpolation of the fields `what` selects (0: q(1..4); 1: the
 * turbulence scalars, nu_tilde or k and omega) to out, point-major,
 * desalm_ov_list_fields(l, what) values per point; without weights they are
 * donee nodes and desalm_ov_list_scatter writes in's values into them.  out
 * and in are device memory of the blocks' GPU; each call returns when its
 * kernel is done, ordered after the blocks' queued work and before their
 * next.  A host cell must have all eight corners in its block.  Which points
 * go to which rank, and the transfer itself (NCCL), are the caller's: see
 * desalm/overset_dist.py. */
typedef struct desalm_ov_list desalm_ov_list;
int  desalm_ov_list_create(desalm_ctx* const* ctxs, int nctx, int n, const int* pts, const double* coef,
                           desalm_ov_list** out);
void desalm_ov_list_destroy(desalm_ov_list* l);
const char* desalm_ov_list_last_error(const desalm_ov_list* l);
int  desalm_ov_list_fields(const desalm_ov_list* l, int what);
int  desalm_ov_list_gather(desalm_ov_list* l, int what, double* out);
int  desalm_ov_list_scatter(desalm_ov_list* l, int what, const double* in);

/* Kernel of each level's DAF line sweeps, nl[3 * level + direction]
 * (directions i, j, k; 0 for levels the case does not have):
 *   2  lines of at most 32 rows: warp-shuffle cyclic reduction, one warp per
 *      line system (always chosen for such lines; it eliminates in another
 *      order, so its values agree with the others' to rounding);
 *   1  the lines-in-lanes Thomas kernel (each warp solves 32 lines, the
 *      eliminated rows kept in a global scratch);
 *   16, 8, 4  the shared-memory slab Thomas kernel with that many lines per
 *      CTA;
 * for longer lines the Thomas kernel timed fastest on this GPU when the grid
 * was set (desalm_set_grid tries each), or 0 where the timing is off
 * (environment DESALM_AUTOTUNE=0): cyclic reduction for short lines, the
 * lines-in-lanes kernel for the others.  The Thomas kernels do the same
 * operations in the same order: choosing among them changes the time only. */
int  desalm_sweep_widths(desalm_ctx* ctx, int nl[12]);
/* The same for the turbulence model's line sweeps of the fine level,
 * nl[direction]: 1 lines in lanes, 32, 16 or 8 slab lines per CTA, 0 the
 * default (lines in lanes).  The i and j sweeps are timed; the k sweep takes
 * the j sweep's choice. */
int  desalm_turb_sweep_widths(desalm_ctx* ctx, int nl[3]);
/* Sets the kernels of the line sweeps (values as above; nl or turb may be
 * NULL to leave that set alone).  A slab width whose shared memory does not
 * fit, 2 for lines longer than 32 rows, or a width for a level the case does
 * not have, is DESALM_EINVAL and changes nothing.  Setting the grid again
 * re-times them. */
int  desalm_set_sweep_widths(desalm_ctx* ctx, const int nl[12], const int turb[3]);
/* CTA tile (threads along i, j, k; 128 in all) of each level's residual
 * kernels, tiles[9 * level + 3 * kernel + axis], kernel 0 = the first
 * residual pass (K_R), 1 = the recalculated residual, 2 = the SA residual
 * (fine level only; the k-omega residual has a fixed tile of 31 x 4 x 2
 * nodes): timed at eight tiles when the grid is set and the fastest kept, or
 * 32 x 4 x 1 where the timing is off (DESALM_AUTOTUNE=0).  Each K_R thread
 * computes two nodes, k planes apart by the tile's k extent.  Kernels 0 and
 * 1 are also timed as the face-shared kernel, reported as the tile
 * 31 x 4 x 2 (256 threads, each viscous face flux formed once for the two
 * nodes beside it).  The tile changes the time only: every node is computed
 * by the same operations. */
int  desalm_kernel_tiles(desalm_ctx* ctx, int tiles[36]);
/* One pseudo-time iteration of the loop above (for callers that drive the
 * loop themselves); rep->residual receives the iteration's residual. */
int  desalm_pseudo_iteration(desalm_ctx* ctx, desalm_step_report* rep);
/* Wait for all work on the context's stream. */
int  desalm_sync(desalm_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events with the library's. */
void* desalm_stream(desalm_ctx* ctx);

/* Instrumentation.  desalm_profile(ctx, 1) brackets every kernel launch with
 * CUDA events on the context stream and resets the statistics and the launch
 * counter; desalm_kernel_stats() returns, per kernel class and level
 * (desalm_kernel_class_count() x 4 entries, index class*4 + level-1), the
 * accumulated milliseconds, launches and nodes processed, plus the total
 * number of kernels launched since the reset. */
int  desalm_profile(desalm_ctx* ctx, int enable);
int  desalm_kernel_stats(desalm_ctx* ctx, double* ms, long* launches,
                         double* nodes, long* total_launches);
int  desalm_kernel_class_count(void);

/* No counterpart in the reference.  desalm_mg_residual for callers that
 * cannot allocate device memory: Fortran drivers whose device arrays belong
 * to another runtime or pool allocator that must see every allocation, and
 * processes held to a fixed device-memory budget.  It gives the same five
 * log10 mean |q - qold| values over the interior of an im x jm x km level,
 * from caller-owned device arrays q and qold (five fields of im*jm*km
 * doubles each, field-major, i fastest), written to the host array res; the
 * call waits for its own work on `stream` before it returns.  It calls no
 * cudaMalloc, cudaFree or allocating library routine: its scratch is a fixed
 * device array of about 2.5 MiB that every GPU loading the library holds
 * until exit.  Grids with more than 134,217,728 interior nodes (512^3) do not
 * fit it and are rejected with DESALM_ENOMEM before any work is queued;
 * null arrays give DESALM_EINVAL.  Calls share the scratch, so calls that
 * overlap on the GPU race.  The first call on each device, with that device
 * current, looks up the scratch's device address and keeps it for the
 * process: make that first call before any stream capture, and do not call
 * cudaDeviceReset after it.  stream may be NULL (the legacy default
 * stream). */
int  desalm_mg_residual_noalloc(const double* q, const double* qold, int im,
                                int jm, int km, double res[5], void* stream);

/* ---------------------------------------------------------------------
 * Learned initial guess (predictor DESALM_PRED_LEARNED).  The reference
 * starts each physical step from q^n (src/mg_driver.F90:48-51); these calls
 * extend that step.  A 4-layer 3x3x3 convolutional network (15 -> 32 -> 32 ->
 * 32 -> 5 channels, ReLU, zero padding, BF16 activations and weights, FP32
 * accumulation) maps, per fine node, q^n, q^n - q^{n-1} and q^{n-1} - q^{n-2}
 * of (p, u, v, w, nu_tilde), each divided by its RMS over the grid, to
 * (q^{n+1} - 2 q^n + q^{n-1}) / s_f, s_f the RMS of (q^n - q^{n-1})_f.  At
 * the start of every physical step desalm_begin_step trains it on the step
 * just converged (train_steps Adam steps on the mean squared error) and, once
 * it has seen warm samples, starts the pseudo-time loop from
 * 2 q^n - q^{n-1} + s_f * alpha_f * output; a node whose output is not
 * finite keeps the linear extrapolation.  alpha_f, the blend, is by default
 * the least-squares factor <y_f, t_f> / <y_f, y_f> limited to [0, 1], where
 * y is the network's output on the newest sample before it trains on it and
 * t that sample's target: a network that does not help gets alpha near 0 and
 * leaves the linear guess.  The scales are those of the time levels at hand; a
 * difference whose RMS is below 1e-12 of its field's RMS has scale zero, so
 * that field gets no correction.  desalm_mg_driver restarts a step begun from
 * the network's guess from the linear guess when the step ends with a
 * non-finite norm or a zero pivot, and then uses the network again only after
 * warm more samples.
 *
 * Flat parameter vector (FP32): for each layer W[cout][cin][27] with the
 * stencil offset o = (dk+1)*9 + (dj+1)*3 + (di+1), then b[cout].
 * --------------------------------------------------------------------- */
typedef struct desalm_lp_report {
  long nparam;        /* parameters (72,677)                              */
  long samples;       /* time levels trained on                           */
  long train_steps;   /* Adam steps taken                                 */
  long predictions;   /* physical steps started from the network's guess  */
  long fallbacks;     /* of those, restarted from the linear guess after a
                         non-finite norm or a zero pivot                  */
  double first_loss;  /* loss of the first training step (-1: none yet)   */
  double last_loss;   /* loss of the latest training step                 */
  double heldout_ratio; /* on the newest sample, before training on it: the
                         squared error of the blended correction over that
                         of no correction (the linear guess); < 1 means
                         the network helps (-1: no sample yet)            */
  double alpha[5];    /* current blend of each field's correction         */
} desalm_lp_report;

/* buffers readable with desalm_lp_get_buffer */
#define DESALM_LP_FEATURES 0   /* [16][N] scaled inputs of the latest pass (channel 15 zero) */
#define DESALM_LP_TARGET   1   /* [5][N] latest training target                          */
#define DESALM_LP_OUTPUT   2   /* [5][N] latest network output (FP32)                    */
#define DESALM_LP_SCALES   3   /* [16] reciprocal RMS of the 15 input channels (0: still) */
#define DESALM_LP_ALPHA    4   /* [5] blend of each field's correction                   */

/* Settings; a negative value keeps the current one.  Defaults: 8 Adam steps
 * per sample, warm = 2 samples before the first guess, lr = 1e-3, and
 * ymax = 8: the output used in the guess is limited to [-ymax, ymax]. */
int  desalm_lp_config(desalm_ctx* ctx, int train_steps, int warm, float lr,
                      float ymax);
int  desalm_lp_report_get(desalm_ctx* ctx, desalm_lp_report* r);
/* Blend: alpha < 0 (default) automatic; 0 <= alpha <= 1 fixed for every field. */
int  desalm_lp_blend(desalm_ctx* ctx, float alpha);
/* Which fields take the network's correction: bit f of mask for field f
 * (p, u, v, w, nu_tilde); the others keep the linear extrapolation.
 * Default 0 (no field): the linear extrapolation of converged time levels
 * satisfies the discrete equations to second order in dt, and a pointwise
 * correction of any field breaks that consistency, which the
 * artificial-compressibility iteration relaxes slowly (every correction
 * measured raised the pseudo-iterations per step).  The network still trains
 * on every step; desalm_lp_report_get gives its held-out error. */
int  desalm_lp_fields(desalm_ctx* ctx, int mask);
/* nparam floats in the flat layout above; set restarts the Adam moments */
int  desalm_lp_get_params(desalm_ctx* ctx, float* theta);
int  desalm_lp_set_params(desalm_ctx* ctx, const float* theta);
/* One forward pass on host features x [16][N] (fine-level node order,
 * i fastest) giving y [5][N]; with a target t [5][N] also the loss
 * mean((y - t)^2) and its gradient with respect to the flat parameters.
 * y, loss and grad may be NULL.  Changes no parameter. */
int  desalm_lp_eval(desalm_ctx* ctx, const float* x, const float* t, float* y,
                    double* loss, float* grad);
int  desalm_lp_get_buffer(desalm_ctx* ctx, int which, float* out);

/* ---------------------------------------------------------------------
 * Actuator-line forcing (the reference's rhs_lines, src/rhs_lines.F90:47-483,
 * called inside solver_daf on the fine level when turbines are on,
 * src/solver_daf.F90:378-381).  The driver computes the geometry tables the
 * reference's init_lines builds (src/init.F90:1156-1710) and passes them once;
 * every fine-level DAF step then, on the GPU, interpolates the velocity at each
 * blade element, looks up lift and drag in the airfoil polars, forms the
 * element forces and projects them with a Gaussian kernel onto the kernel
 * nodes, adding them to rh(2:4) before the modal transforms.  The
 * recalculated residual (src/solver_daf.F90:432-463) does not call rhs_lines
 * and gets no forcing.  Indices are 1-based global (i, j, k) as in the
 * reference; arrays are copied at desalm_alm_set.  As in the reference, a
 * polar lookup that finds no interval keeps the previous element's values,
 * and elements or kernel nodes whose cell is not interior are skipped.
 * Differences: the forcing acts on the fine level only (the reference also
 * calls rhs_lines on coarse levels with fine-grid indices, which is
 * meaningful only without coarsening); an azimuth that rounds to one bin past
 * the last wraps to the first (the reference reads past its table); the
 * polars come in arrays instead of the airfoil files the reference reopens
 * for every element; its per-element prints are not reproduced.  Two
 * turbines whose kernel lists share a node add to it in either order.
 * --------------------------------------------------------------------- */
typedef struct desalm_alm_turbine {
  int nblades, nelems, nangles;  /* nangles azimuth bins: dtheta_interp = 2 pi / nangles */
  double tsr;                     /* tip-speed ratio                                    */
  double tur_rad, hub_rad;        /* rotor and hub radius (m)                           */
  double angle;                   /* azimuth of blade 1 (rad); desalm_alm_set_angle     */
  /* element cells per azimuth bin, entry e = (nang - 1) * nelems + (elem - 1):
   * node_index[3 e + 0..2] = i, j, k of the cell's lower corner;
   * node_pos[27 e + 0..26] = xf, yf, zf, then the corners 000, 100, 110, 010,
   * 001, 101, 111, 011 as x, y, z each (node_indexes_pos(...,1:27)) */
  const int* node_index;
  const double* node_pos;
  /* per fine-grid (j, k), index (j - 1) + jm (k - 1): disk_dat[8 index + c]
   * = radius, area, theta, dV, chord, twist, inter, relthick (the reference's
   * disk_dat(j, k, 1:8)); polar_b / polar_a = the airfoil polar before / after */
  const double* disk_dat;
  const int* polar_b;
  const int* polar_a;
  /* kernel nodes: nker entries; ker_index[3 n] = i, j, k; ker_pos[3 n] = x, y,
   * z; ker_dat[4 n] = radius, area, theta, dV (disk_dat_ker(i, j, k, 1:4)) */
  int nker;
  const int* ker_index;
  const double* ker_pos;
  const double* ker_dat;
} desalm_alm_turbine;

typedef struct desalm_alm {
  int n_tur;
  const desalm_alm_turbine* tur;
  double vel_infty;               /* free-stream velocity (m/s): omega = vel_infty tsr / tur_rad */
  double length_scale;            /* m per grid unit; vel_scale = ren 1e-6 / length_scale        */
  /* airfoil polars as the reference's airfoil files hold them: table p has
   * polar_count[p] rows (angle in degrees, Cl, Cd) at polar_rows[3 (polar_offset[p] + r)];
   * its last row has angle -999, the end marker */
  int npolar;
  const int* polar_offset;
  const int* polar_count;
  const double* polar_rows;
} desalm_alm;

/* Turns the forcing on for this context (n_tur = 0 turns it off).  Every
 * element cell and kernel node must be an interior fine node (the cell's
 * upper corner included), every polar index valid. */
int  desalm_alm_set(desalm_ctx* ctx, const desalm_alm* alm);
/* The azimuth of turbine n_t (1-based); the driver advances it once per
 * physical step, as src/main.F90:42-50 does. */
int  desalm_alm_set_angle(desalm_ctx* ctx, int n_t, double angle);
/* After a fine-level DAF step: what = 0, the element forces of the last call
 * as (xf, yf, zf, fx, fy, fz) per element, turbines, blades, elements in
 * that order (forces_lines); what = 1, the force added to rh(2:4), [3][N]
 * over the fine level. */
#define DESALM_ALM_FORCES 0
#define DESALM_ALM_FIELD  1
int  desalm_alm_get(desalm_ctx* ctx, int what, double* out);

/* ---------------------------------------------------------------------
 * Synthetic inflow turbulence: the random flow generator of Smirnov, Shi &
 * Celik (2001) that the reference runs when rfgt is set
 * (src/global_param.F90:135; src/rfg_inlet.F90, src/rfg.F90).  Before each
 * physical step the driver sets the velocities of the inflow plane i = 1,
 * j = 2..jm-1, k = 2..km-1 to
 *   q(2:4) = um + M diag(c) sqrt(2/N) sum_n [p_n cos(a_n) + q_n sin(a_n)],
 *   a_n = (k_n upsilon / c) . (x / eta) + omega_n t / tau,  upsilon = eta / tau,
 * with M diag(c^2) M^T the node's velocity correlation tensor, tau and eta its
 * time and length scales.  The tables are those of the reference's
 * inlet.bin.dat (rfg_um, rfg_uij, rfg_t_ts, rfg_t_ls over the fine (j, k)
 * plane, Fortran layout) and of initialize_rfg (p_rfg, q_rfg, k_rfg,
 * omega_rfg).  Hold the plane with an inflow face (btype(1) = 4).
 * Differences: every node's tensor is decomposed once at desalm_rfg_set (the
 * reference repeats it at every step), by Jacobi rotations with each
 * eigenvector's largest component positive (the reference keeps the signs
 * LAPACK ssyev returns); FP64 (the reference: real(rdf) = FP32).
 * --------------------------------------------------------------------- */
typedef struct desalm_rfg {
  int nmodes;              /* N: spectrum samples (rfg_inlet_seed.dat), 0 turns it off */
  const double* p;         /* p_rfg(3, N): p[3 n + d]                                   */
  const double* q;         /* q_rfg(3, N)                                               */
  const double* k;         /* k_rfg(3, N)                                               */
  const double* omega;     /* omega_rfg(N)                                              */
  const double* um;        /* rfg_um(3, jm, km): um[3 (j + jm k) + d], 0-based j, k      */
  const double* uij;       /* rfg_uij(6, jm, km): r11, r12, r13, r22, r23, r33           */
  const double* t_ts;      /* rfg_t_ts(jm, km): time scale tau                          */
  const double* t_ls;      /* rfg_t_ls(jm, km): length scale eta                        */
} desalm_rfg;

/* initialize_rfg (src/rfg.F90:42-96) on the host: draws zeta, xi ~ N(0, 1)
 * (3 N each), k ~ N(0, 0.5^2) (3 N), omega ~ N(0, 1) (N) in the reference's
 * order and forms p = zeta x k, q = xi x k.  The normal deviates come from the
 * polar method over a splitmix64 stream seeded by `seed`, not from the
 * reference's generator, so a seed gives other samples of the same
 * distribution.  1 <= nmodes <= 2^20.  Needs no GPU. */
int  desalm_rfg_modes(int nmodes, long long seed, double* p, double* q, double* k, double* omega);
/* rfg_init (src/rfg_inlet.F90:47-105): copies the tables to the device and
 * decomposes every inflow node's correlation tensor.  Needs the grid
 * (DESALM_ENOTREADY before desalm_set_grid); a later desalm_set_grid turns
 * the generator off until it is set again.  DESALM_EINVAL when a tensor is
 * not positive definite or a scale is not positive.  NULL or nmodes = 0
 * turns the generator off. */
int  desalm_rfg_set(desalm_ctx* ctx, const desalm_rfg* rfg);
/* rfg_mpi_inlet_forcing (src/rfg_inlet.F90:107-173) for physical time `time`:
 * sets q(2:4) of the inflow plane on the device, ordered on the context's
 * stream.  Call it before desalm_mg_driver / desalm_begin_step, as
 * src/main.F90:60 does; the step then shifts the plane into q^n like the rest
 * of q, and when the guess is extrapolated or learned, forces the plane again
 * for the same time after the guess, so the step holds the forced values.
 * A desalm_set_state between the two calls replaces the forced plane like the
 * rest of q; the extrapolated or learned guess still forces it again. */
int  desalm_rfg_inlet(desalm_ctx* ctx, double time);

/* Self-test of the device watchdog: a kernel waits, through the same bounded
 * wait as the tensor-core kernels, on a barrier that nothing completes, for
 * `seconds` (<= 10); the call returns DESALM_ETIMEOUT when the wait gave up
 * and reported it, as it must.  No counterpart in the reference. */
int  desalm_watchdog_selftest(desalm_ctx* ctx, double seconds);

/* ---------------------------------------------------------------------
 * On-disk formats of the reference, for drivers that run real cases and
 * checkpoint from the device.  Grid and solution files are Fortran
 * unformatted sequential files (each record: 4-byte little-endian byte count,
 * payload, the count again) of FP32 values, i fastest, one block.  Host arrays
 * use this header's layouts: q and qn as (1:5, i, j, k) with the component
 * fastest, x, y, z, wd and nu_t as (i, j, k).  me = 4 for a laminar case, 5
 * with Spalart-Allmaras (q(5) = nu_tilde).  These functions make no CUDA call;
 * on failure they return DESALM_EIO (or DESALM_EINVAL) and
 * desalm_io_error() describes it.
 * --------------------------------------------------------------------- */
const char* desalm_io_error(void);

/* 'grid' (src/init.F90:2226-2243): records x, y, z and, when turbulent, the
 * wall distance wd. */
int  desalm_grid_read(const char* path, int im, int jm, int km, int turbulence,
                      double* x, double* y, double* z, double* wd);
int  desalm_grid_write(const char* path, int im, int jm, int km, int turbulence,
                       const double* x, const double* y, const double* z,
                       const double* wd);

/* Restart file.  Write (output_restart, src/main.F90:315-393): one record each
 * of q(1..me), then nu_t when turbulent, then qn(1..me).  Read (init_solu,
 * src/init.F90:2324-2475): the same records; for a laminar case the reference
 * reads q(1..me) as one record of me*N values and then qn likewise, and both
 * laminar layouts are accepted here.  Components past me read as zero; nut may
 * be NULL. */
int  desalm_solu_write(const char* path, int im, int jm, int km, int turbulence,
                       const double* q, const double* qn, const double* nut);
int  desalm_solu_read(const char* path, int im, int jm, int km, int turbulence,
                      double* q, double* qn, double* nut);

/* 'filestat' (src/main.F90:374-381 writes, src/init.F90:268-276 reads):
 * list-directed text, time and step, then one turbine angle a line; reading
 * brings an angle >= 2 pi back by 2 pi, as the reference does. */
int  desalm_filestat_write(const char* path, double time, int ntime,
                           const double* angle, int n_tur);
int  desalm_filestat_read(const char* path, double* time, int* ntime,
                          double* angle, int n_tur);

/* The context's device state to / from a restart file (layouts above).
 * After a read, q^{n-1} is zero, as after the reference's restart
 * (src/init.F90:1089); the next physical step's history shift refills it. */
int  desalm_checkpoint_write(desalm_ctx* ctx, const char* path);
int  desalm_checkpoint_read(desalm_ctx* ctx, const char* path);
/* The learned guess's parameters, Adam moments and counters (a format of
 * this library; the reference has no network). */
int  desalm_lp_checkpoint_write(desalm_ctx* ctx, const char* path);
int  desalm_lp_checkpoint_read(desalm_ctx* ctx, const char* path);

#ifdef __cplusplus
}
#endif
#endif /* DESALM_H */
