/*
 * itlbm.h -- C ABI of the B200 colour-gradient lattice-Boltzmann step.
 *
 * One time step is: D3Q19 with one node in z, periodic all-fluid slab, BGK with Guo forcing,
 * Latva-Kokko--Rothman recolouring, the mediator isotropic gradient of rho^N and one of seven
 * interfacial-tension operators (P1, P3 chi, F1, F2, F3 xi).  Every entry point below replaces one
 * piece of the reference's stepping loop or of its operator seam; the reference file:line each one
 * stands in for is given beside it (paths relative to the reference project root).
 *
 * Conventions
 *   - Plain C types only.  A `stream` argument is a cudaStream_t passed as void* (NULL = legacy
 *     default stream).  Calls marked "async" only enqueue work on that stream.
 *   - Every int-returning call returns ITLBM_OK (0) or a negative ITLBM_E_* code; the text of the
 *     last failure on the calling thread is returned by itlbm_last_error().  No call traps or hangs
 *     the device: waits are bounded and report ITLBM_E_TIMEOUT.
 *   - The library owns all device memory of a case.  Populations handed across the ABI are FP64 in
 *     the reference's array-of-structures order, f[pto * 19 + i] with pto = x + nx * y, exactly the
 *     layout of LATTICE::inif_R / inif_B (SimBoltz_Functions/Definitions.cpp:52-114).
 *   - Lattice order of the 19 velocities is that of def_lattice_d3q19
 *     (SimBoltz_Functions/LBM_functions.cpp:366-497).
 */
#ifndef ITLBM_H
#define ITLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ITLBM_NVEL 19
#define ITLBM_N_ANG 256          /* rays of the interface-mode measure (Operadores_tensao.cpp:385) */

/* ---- return codes ------------------------------------------------------------------------- */
enum {
    ITLBM_OK          =  0,
    ITLBM_E_ARG       = -1,   /* invalid argument                                               */
    ITLBM_E_OOM       = -2,   /* device or host allocation failed                              */
    ITLBM_E_CUDA      = -3,   /* CUDA runtime error                                            */
    ITLBM_E_NODEVICE  = -4,   /* no usable CUDA device                                         */
    ITLBM_E_NONFINITE = -5,   /* non-finite state found                                        */
    ITLBM_E_ADMISSION = -6,   /* batch: request does not fit the HBM budget or slot table      */
    ITLBM_E_TIMEOUT   = -7,   /* a bounded wait expired                                        */
    ITLBM_E_PARSE     = -8,   /* input text could not be parsed                                */
    ITLBM_E_IO        = -9,   /* file could not be opened or written                           */
    ITLBM_E_STATE     = -10   /* call not valid in the object's current state                  */
};

/* ---- tension operator: OPERADOR (Operadores_tensao.cpp:45-59) ------------------------------ */
enum {
    ITLBM_OP_P1 = 1,          /* OP_P1 : weighted Gunstensen perturbation, lambda = 0           */
    ITLBM_OP_P3 = 3,          /* OP_P3 : Liu-Valocchi-Kang family B_i(chi), lambda = 1          */
    ITLBM_OP_F1 = 11,         /* OP_F1 : CSF force (sigma/2) kappa grad rho^N                   */
    ITLBM_OP_F2 = 12,         /* OP_F2 : divergence of the capillary stress                    */
    ITLBM_OP_F3 = 13          /* OP_F3 : chemical-potential force mu grad rho^N                 */
};

typedef struct itlbm_operador {
    int    tipo;              /* ITLBM_OP_*                                                     */
    double chi;               /* P3 only; default 0.5                                          */
    double xi;                /* F3 only; default 1.569988                                     */
    char   nome[16];          /* the operator word as read ("P1", "P3", ...)                   */
} itlbm_operador;

/* ---- case description --------------------------------------------------------------------- */
enum { ITLBM_GEOM_DROP = 0, ITLBM_GEOM_STRIP = 1 };
/* ITLBM_PREC_F32_FOLD (no counterpart in the reference): FP32 storage of the nine in-plane classes of
 * D3Q19 per colour (144 instead of 304 bytes per update).  For the one-node slab the class sums evolve
 * exactly as the 19 populations do (up to rounding); read_pops returns each class split among its
 * members by weight, so the per-direction minima and counts of negative populations and the P_zz of the
 * strip's sigma_pop are those of the split. */
enum { ITLBM_PREC_F64 = 0, ITLBM_PREC_F32 = 1, ITLBM_PREC_F32_FOLD = 2 };

typedef struct itlbm_case_desc {
    int    nx, ny;            /* box nx x ny x 1, all fluid, periodic                           */
    itlbm_operador op;
    double tau;               /* single BGK time (tau_R == tau_B), data_in.txt                 */
    double beta;              /* recolouring factor (recoll)                                    */
    double A_fact;            /* amplitude A (P class) or sigma (F class): fat_R_B             */
    double rho_R, rho_B;      /* initial densities of the pure fluids                          */
    int    geometry;          /* ITLBM_GEOM_DROP (Imm_OPS) or ITLBM_GEOM_STRIP (Imm_INCL)       */
    double radius;            /* drop radius; <= 0 selects nx / 4 (Imm_OPS.cpp:134)            */
    double k_profile;         /* logistic slope of the initial drop; <= 0 gives a sharp step   */
    double v0;                /* drop: uniform initial velocity along x (velocity.txt)         */
    int    p, q;              /* strip: interface normal (p, q) (inclinacao.txt)               */
    int    precision;         /* ITLBM_PREC_F64 (plain) or ITLBM_PREC_F32 (shifted storage)    */
} itlbm_case_desc;

/* ---- diagnostics of a drop: DROP + GI_DATA + MODOS ---------------------------------------- */
/* Fields follow DROP (SimBoltz_Functions/Definitions.cpp:251-339), GI_DATA
 * (Galilean_diagnostics.cpp:7-16) and MODOS (Operadores_tensao.cpp:380). */
typedef struct itlbm_drop_diag {
    int       ok;             /* calc_galilean's return value                                  */
    int       step;
    /* DROP */
    double    x0, y0, area, raio, raio_grad, raio_linha;
    double    massa_R, massa_B, qx, qy, qz, u_max, u_rms;
    double    p_in, p_out, sd_in, sd_out, delta_p, sigma, p_centro, p_canto, sigma_linha;
    double    K_perfil, r_perfil, res_perfil, esp_perfil;
    int       n_perfil, n_in, n_out, n_fluid, n_ruim;
    /* GI_DATA */
    double    mean_x, mean_y, mean_z, drop_x, drop_y;
    double    max_ref, rms_ref, max_mean, rms_mean, max_lab, rms_lab;
    double    min_f, min_rho, min_phi, max_phi, axis_ratio, center_dx, center_dy, x_unwrapped;
    long long negative_total, negative_color;
    int       bad;
    /* MODOS */
    double    R0, a2, a4, a8, rmin, rmax;
} itlbm_drop_diag;

/* ---- diagnostics of an inclined strip: INCL (Imm_INCL.cpp:62-70) --------------------------- */
typedef struct itlbm_strip_diag {
    int       ok;
    int       step;
    double    sigma_pop, int_grad, K, res, d0;
    double    u_max, u_rms, un_max, ut_max;
    double    massa_R, massa_B, qx, qy;
    double    min_f, SFx, SFy;
    long long neg_total, neg_cor;
    int       n_ruim, n_ajuste;
} itlbm_strip_diag;

typedef struct itlbm_case itlbm_case;

/* ---- library ----------------------------------------------------------------------------- */
const char *itlbm_version(void);
const char *itlbm_strerror(int code);
const char *itlbm_last_error(void);
int         itlbm_device_count(int *count);

/* le_operador (Operadores_tensao.cpp:66-86): one line "<P1|P3|F1|F2|F3> [chi|xi]".  The _read form
 * reads the first line of a file; the _parse form takes the text itself.  ITLBM_E_PARSE when the
 * word is unknown or missing (the reference's `return false`). */
int itlbm_operador_parse(const char *text, itlbm_operador *op);
int itlbm_operador_read(const char *path, itlbm_operador *op);

/* ---- one case ---------------------------------------------------------------------------- */
/* Allocates the double-buffered state on the current device and seeds it:
 *   drop  -> initial_conditions_drop (SimBoltz_Functions/Initial_conditions.cpp:37-169) with the
 *            centre (nx/2, ny/2), EQ_CLASSICO, as called at Imm_OPS.cpp:199-202;
 *   strip -> the logistic strip of Imm_INCL.cpp:309-334.
 * Replaces the allocation and set-up block Imm_OPS.cpp:156-202 / Imm_INCL.cpp:268-334. */
int  itlbm_case_create(const itlbm_case_desc *desc, itlbm_case **out);
void itlbm_case_destroy(itlbm_case *c);

enum { ITLBM_STEP_KEEP_AUX = 1 };   /* keep F and |grad rho^N| of the last step for diagnostics */

/* Async.  Runs `nsteps` time steps, each one the body of the loop Imm_OPS.cpp:252-287 (mediator
 * emission and streaming, calcula_forca, colisao_comum, propag_site, buffer swap).  With
 * ITLBM_STEP_KEEP_AUX the force and the mediator gradient of the LAST step are kept for the
 * diagnostics below (the reference's `forca` array and inif_m at its diagnostic point). */
int  itlbm_case_step(itlbm_case *c, int nsteps, int flags, void *stream);
int  itlbm_case_sync(itlbm_case *c);
long long itlbm_case_steps_done(const itlbm_case *c);

/* Sync.  The drop measures of one diagnostic step (Imm_OPS.cpp:299-304): calc_galilean
 * (Galilean_diagnostics.cpp:24-105) with calc_laplace_tension / calc_drop_radius
 * (SimBoltz_Functions/Other_functions.cpp:60-276, 453-554), calc_perfil_logistico
 * (Other_functions.cpp:318-448) and modos_interface (Operadores_tensao.cpp:382-449).  They read the
 * post-collision populations of the last step, as the reference does; `step` is that step's index
 * and (x_ini, y_ini) the initial centre.  The last step must have run with ITLBM_STEP_KEEP_AUX when
 * the operator is of class F. */
int  itlbm_case_diag_drop(itlbm_case *c, int step, double x_ini, double y_ini, itlbm_drop_diag *out,
                          void *stream);

/* No counterpart in the reference.  itlbm_case_diag_drop without any allocation, for callers that
 * must not touch the CUDA allocator: a serving process whose HBM is all committed to its case pool,
 * or a monitor thread beside a running batch, where the lazy cudaMalloc of the scratch could fail
 * and a cudaFree would synchronize the whole device.  Same kernels, same results.
 *   - The scratch is one fixed device array of 14 MiB per device, so the case may have at most
 *     ITLBM_STATIC_DIAG_MAX_NODES nodes and sides of at most ITLBM_STATIC_DIAG_MAX_SIDE; larger
 *     cases get ITLBM_E_ARG (use itlbm_case_diag_drop).
 *   - The first call on a device looks the array's address up (cudaGetSymbolAddress, with that
 *     device current); make it before any stream capture begins.  Under CUDA's lazy module loading
 *     (the default since CUDA 12.2) that first call is also when the device commits the array's
 *     14 MiB, so make it while the device still has that much free, before a case pool takes the
 *     rest of its memory.
 *   - Nothing has to start at zero: every call clears what it accumulates into.
 *   - Calls that overlap in time on the same device (from several host threads) share the scratch
 *     and race; serialize them.  A call returns only after its stream is synchronized. */
#define ITLBM_STATIC_DIAG_MAX_NODES 262144  /* 512 x 512 */
#define ITLBM_STATIC_DIAG_MAX_SIDE  4096
int  itlbm_case_diag_drop_static(itlbm_case *c, int step, double x_ini, double y_ini,
                                 itlbm_drop_diag *out, void *stream);

/* Sync.  mede_inclinada (Imm_INCL.cpp:85-189) on the post-collision populations of the last step,
 * which must have run with ITLBM_STEP_KEEP_AUX. */
int  itlbm_case_diag_strip(itlbm_case *c, int step, itlbm_strip_diag *out, void *stream);

/* Sync.  Copies populations to host, FP64, reference AoS order.  which = 0: the state at the top of
 * the next step (inif_R / inif_B after the swap at Imm_OPS.cpp:368-371); which = 1: the
 * post-collision populations of the last step (inif_R / inif_B at the diagnostic point
 * Imm_OPS.cpp:293).  FP32 cases are reconstructed to FP64. */
int  itlbm_case_read_pops(itlbm_case *c, int which, double *fR, double *fB);

/* Sync.  Overwrites the state at the top of the next step (same layout as read_pops which = 0). */
int  itlbm_case_write_pops(itlbm_case *c, const double *fR, const double *fB);

/* The two forms of the per-node velocity that the reference's output files carry. */
enum {
    ITLBM_FIELDS_VTK = 0,     /* vel_*.vtk, rec_velocity (LBM_functions.cpp:1349-1458): the colour    */
                              /* velocities of calcula weighted by the concentrations, u = c_R u_R +  */
                              /* c_B u_B, minus (F/2)/rho for a case with a force                       */
    ITLBM_FIELDS_PROFILE = 1  /* perfil.dat, mede_inclinada (Imm_INCL.cpp:104-162): the mixture       */
                              /* momentum, u = (sum_i f_i c_i - F/2) / rho (NaN where !(rho > 0))      */
};

/* Sync.  Per-node fields of the post-collision populations of the last step, each nx*ny doubles in
 * pto order (any pointer may be NULL): rho_R and rho_B (rec_density, LBM_functions.cpp:1457-1511),
 * the velocity of vel_*.vtk (ITLBM_FIELDS_VTK: rec_velocity, LBM_functions.cpp:1349-1458, the Guo
 * half-force removed) and the force of the last step (`forca`, Imm_OPS.cpp:174-181), 3 per node.
 * In FP64 every value is the reference's, rounded as the reference rounds it. */
int  itlbm_case_read_fields(itlbm_case *c, double *rho_R, double *rho_B, double *ux, double *uy,
                            double *uz, double *force);
/* Sync.  The per-node values perfil.dat prints (Imm_INCL.cpp:101-162): rho_R, rho_B and the
 * ITLBM_FIELDS_PROFILE velocity (ux, uy), post-collision populations of the last step. */
int  itlbm_case_read_profile(itlbm_case *c, double *rho_R, double *rho_B, double *ux, double *uy);

/* Sync.  Case snapshots: the reference restarts an interrupted batch from step 0 (rodar_lote.py:5-7);
 * these save a case (its description, its step count and its populations at the top of its next
 * step, in its own precision) and restore it on the current device.  Stepping a restored case gives
 * the same bits the saved case would have given.  The kept force (ITLBM_STEP_KEEP_AUX) is not saved:
 * the next step of a restored class-F case must keep it before a diagnostic. */
int  itlbm_case_save(itlbm_case *c, const char *path);
int  itlbm_case_load(const char *path, itlbm_case **out);
/* The description and step count stored in a snapshot, without touching the device. */
int  itlbm_snapshot_info(const char *path, itlbm_case_desc *desc, long long *steps);

/* ---- batches: many cases stepped together ------------------------------------------------- */
/* The batched form of the loop Imm_OPS.cpp:246-372 / Imm_INCL.cpp:358-442 for many independent
 * cases, replacing the process pool of rodar_lote.py (rodar_lote.py:231-243, :300-318).  Admitted
 * cases keep their state on the device; each advance runs a CUDA graph of persistent step launches
 * over a device-resident tile work table (every case's tiles, FP32 and FP64 cases side by side),
 * stops every case at its next diagnostic step (every 500 steps and the last, Imm_OPS.cpp:293),
 * measures it there and retires it at its step count or when it becomes unstable
 * (Imm_OPS.cpp:346-352). */
typedef struct itlbm_batch itlbm_batch;

typedef struct itlbm_batch_config {
    size_t hbm_budget;        /* device bytes the batch may hold; 0 = 90 % of the free memory    */
    int    max_cases;         /* slots; 0 = 4096                                                  */
    int    chunk;             /* steps per graph replay; 0 = 500 (PASSOS_DIAG)                    */
    int    diag_every;        /* diagnostic interval; 0 = 500                                     */
    int    ctas_per_sm;       /* launch shape of the step kernels: < 0 = one CTA per tile of the   */
                              /* work table; > 0 = that many persistent CTAs per SM striding over */
                              /* it; 0 = autotune: the first full replay times the tilings (narrow */
                              /* edge tiles or 32 x 8 throughout) and the two launch shapes        */
                              /* (persistent at the occupancy limit) and keeps the faster of each  */
                              /* (same results)                                                     */
} itlbm_batch_config;

enum { ITLBM_EV_DIAG = 0, ITLBM_EV_DONE = 1, ITLBM_EV_UNSTABLE = 2 };

typedef struct itlbm_batch_event {
    long long tag;            /* the caller's tag of the case                                     */
    int       kind;           /* ITLBM_EV_*                                                        */
    int       geometry;       /* ITLBM_GEOM_* : which of drop / strip is filled                    */
    int       step;           /* step index of the diagnostic (DIAG) or steps run (DONE/UNSTABLE) */
    double    t_submit, t_event;  /* seconds on the batch clock                                  */
    itlbm_drop_diag  drop;
    itlbm_strip_diag strip;
} itlbm_batch_event;

typedef struct itlbm_batch_stats {
    int       active, pending, finished;
    long long node_updates;   /* lattice-node updates done so far                                */
    double    device_ms;      /* device time of the step launches (CUDA events)                  */
    size_t    hbm_used;       /* bytes of case state held                                         */
    int       replays;        /* graph replays so far                                              */
    int       captures;       /* graph (re)captures so far: the work tables changed their grid     */
    double    diag_ms;        /* device time of the diagnostics (CUDA events)                      */
    double    advance_ms;     /* host wall time spent inside itlbm_batch_advance                   */
    double    admit_ms;       /* of which admission: allocation and initial state of new cases     */
    double    capture_ms;     /* of which graph capture and instantiation                          */
    int       launch_mode;    /* launch shape in use: -1 one CTA per tile, 0 persistent CTAs at   */
                              /* the occupancy limit, k > 0 k persistent CTAs per SM               */
    int       held;           /* finished cases kept for itlbm_batch_read_fields (not in `active`) */
    int       narrow_edges;   /* tiling in use: 1 the partial last tile column of a case in 16 x 16 */
                              /* or 8 x 32 tiles, 0 32 x 8 tiles throughout (in the fold, two rows  */
                              /* per thread: 16 x 32, 8 x 64 and 32 x 16); autotuned like the      */
                              /* launch shape; the results do not depend on it                      */
} itlbm_batch_stats;

/* No case memory is allocated until cases are admitted. */
int  itlbm_batch_create(const itlbm_batch_config *cfg, itlbm_batch **out);
void itlbm_batch_destroy(itlbm_batch *b);
/* Queues a case of n_steps steps.  It is admitted at the next advance when its state fits the HBM
 * budget and a slot is free (ITLBM_E_ADMISSION if it can never fit).  `tag` comes back in events. */
int  itlbm_batch_submit(itlbm_batch *b, const itlbm_case_desc *d, int n_steps, long long tag);
/* Batch snapshots (see itlbm_case_save): itlbm_batch_save writes the active case `tag` as it stands
 * between two advances; itlbm_batch_submit_saved queues a case that starts from a snapshot (of a
 * batch or of a single case) and runs on to step n_steps (its diagnostics keep the absolute step
 * numbers). */
int  itlbm_batch_save(itlbm_batch *b, long long tag, const char *path);
int  itlbm_batch_submit_saved(itlbm_batch *b, const char *path, int n_steps, long long tag);
/* One round: admit, run one graph replay (every active case advances to its next diagnostic step
 * or by `chunk` steps), run the diagnostics that fell due, retire finished and unstable cases.
 * Returns the number of events now waiting (>= 0) or an error code. */
int  itlbm_batch_advance(itlbm_batch *b, void *stream);
/* Copies up to `max` waiting events (oldest first) and removes them from the queue. */
int  itlbm_batch_poll(itlbm_batch *b, itlbm_batch_event *ev, int max);
int  itlbm_batch_stats_get(const itlbm_batch *b, itlbm_batch_stats *out);

/* Final fields of batch cases (the files Imm_OPS.cpp:357-364 and Imm_INCL.cpp:101-162 write at the
 * last step).  With itlbm_batch_hold_finished(b, 1), a case that retires (ITLBM_EV_DONE, or
 * ITLBM_EV_UNSTABLE) keeps its state on the device, off the work table and still counted against
 * the HBM budget, until itlbm_batch_release; itlbm_batch_read_fields reads the post-collision fields
 * of its last measured step in the given ITLBM_FIELDS_* form (same values as itlbm_case_read_fields /
 * itlbm_case_read_profile; any pointer may be NULL).  read_fields also accepts an active case whose
 * last advance ended at one of its diagnostic steps.  ITLBM_E_ARG for an unknown tag, ITLBM_E_STATE
 * when the case has no measured step to read. */
int  itlbm_batch_hold_finished(itlbm_batch *b, int on);
int  itlbm_batch_read_fields(itlbm_batch *b, long long tag, int form, double *rho_R, double *rho_B,
                             double *ux, double *uy, double *uz);
int  itlbm_batch_release(itlbm_batch *b, long long tag);

/* ---- operator seam on the device (per-site functions of the reference) -------------------- */
/* Each call copies its host arrays to the device, runs the same device code the step kernel uses,
 * and copies the result back (sync). */

/* perturbacao (Operadores_tensao.cpp:116-133) on n sites: f[k*19+i] += Omega_i(g[k*3..]).  */
int itlbm_dev_perturbacao(const itlbm_operador *op, double A, int n, const double *g, double *f);

/* source (SimBoltz_Functions/LBM_functions.cpp:1603-1673) on n sites: S[k*19+i] from F[k*3..],
 * u[k*3..], rho[k] and tau. */
int itlbm_dev_source(int n, const double *F, const double *u, const double *rho, double tau,
                     double *S);

/* calcula_forca (Operadores_tensao.cpp:202-332) on a periodic nx x ny x 1 field given by its
 * populations (AoS): F[pto*3+a].  sigma is fat_R_B. */
int itlbm_dev_calcula_forca(const itlbm_operador *op, double sigma, int nx, int ny,
                            const double *fR, const double *fB, double *F);

/* colisao_comum (Operadores_tensao.cpp:340-373) on n independent sites: fR, fB (19 per site) are
 * updated in place from the mediator momentum gm[k*3..] (= -grad rho^N) and the force F[k*3..]
 * (ignored for class P).  tau, A_fact and beta as in PARAMETERS. */
int itlbm_dev_colisao_comum(const itlbm_operador *op, double tau, double A_fact, double beta, int n,
                            double *fR, double *fB, const double *gm, const double *F);

#ifdef __cplusplus
}
#endif

#endif /* ITLBM_H */
