/*
 * gpudock.h -- C-ABI of the B200 replica-exchange Monte Carlo (REMC)
 * docking path of GeauxDock / gpudocksm.
 *
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or
 * torch types.  Host buffers are owned by the caller; device memory is owned
 * by the opaque handles (gd_ctx, gd_dcomplex, gd_remc, gd_batch, gd_server).
 * Every call returns gd_status; nothing calls exit().
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   Run()            gpudocksm-rem-1.2/src/run.h:6-17, run.cu:41-353
 *   MonteCarlo_d     gpudocksm-rem-1.2/src/montecarlo_d.cu:59-104
 *   CalcEnergy_d     gpudocksm-rem-1.2/src/calcenergy_d.cu:22-374
 *   ExchangeReplicas gpudocksm-rem-1.2/src/exchangereplicas_d.cu:7-139
 *   OptimizeEnepara  gpudocksm-rem-1.2/src/util.C:405-458
 *   SetTemperature   gpudocksm-rem-1.2/src/util.C:491-532
 *   SetReplica       gpudocksm-rem-1.2/src/util.C:538-558
 *   loadProtein / loadLigand / loadLHM
 *                    gpudocksm-rem-1.2/src/load.C:100-420, 595-990, 1011-1126
 *   loadEnePara / loadWeight / loadNorPara
 *                    gpudocksm-rem-1.2/src/load.C:1139-1419
 *   CalculateSimilarityMatrix
 *                    SimilarityMatirxGen/src/util.C:37-193
 */
#ifndef GPUDOCK_H
#define GPUDOCK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                             */
/* ------------------------------------------------------------------------ */
typedef enum gd_status {
  GD_OK = 0,
  GD_EINVAL = 1,      /* malformed input: sizes, types, indices, NULLs     */
  GD_ENOMEM = 2,      /* host or device allocation failed                   */
  GD_EBUDGET = 3,     /* request larger than the server's HBM budget        */
  GD_ECUDA = 4,       /* a CUDA runtime call failed (see gd_last_error)     */
  GD_ETIMEDOUT = 5,   /* a bounded wait ran out                             */
  GD_ECANCELLED = 6,  /* request cancelled before it finished               */
  GD_ENOTFOUND = 7,   /* unknown request id                                 */
  GD_EAGAIN = 8,      /* not finished yet (poll again)                      */
  GD_ENODEV = 9,      /* no CUDA device / kernel image not loadable         */
  GD_EIO = 10         /* a file could not be read or written                */
} gd_status;

/* Thread-local text of the last error raised on this thread. */
const char *gd_last_error(void);
/* Library version string. */
const char *gd_version(void);

/* ------------------------------------------------------------------------ */
/* Force-field type space: the reference's size.h constants MAXTP1..MAXTP4, */
/* MAXWEI (gpudocksm-rem-1.2/src/size.h:53-75).  These size the parameter   */
/* tables, not the problem, so they stay fixed.                             */
/* ------------------------------------------------------------------------ */
#define GD_NPT 30    /* protein effective-point types (MAXTP1)  */
#define GD_NLT 24    /* ligand atom types (MAXTP2)              */
#define GD_NELE 50   /* electrostatic classes (MAXTP3)          */
#define GD_NRES 20   /* residue types (MAXTP4)                  */
#define GD_NTERM 10  /* energy terms incl. total (MAXWEI)       */
#define GD_NRAW 9    /* un-normalised terms returned in FP64    */

/* MCS coordinate that marks an absent atom (size.h:97). */
#define GD_MCS_INVALID_COORD 728492.0f

/* Energy term order inside a 10-float energy record: the rem order of
 * calcenergy_d.cu:301-309 and dock.h:98-116. */
enum {
  GD_E_VDW = 0, GD_E_ELE = 1, GD_E_PMF = 2, GD_E_PSP = 3, GD_E_HDB = 4,
  GD_E_HPC = 5, GD_E_KDE = 6, GD_E_LHM = 7, GD_E_DST = 8, GD_E_TOTAL = 9
};

/* Raw force field as loaded from the .ff parameter file
 * (EnePara0, gpudocksm-rem-1.2/src/dock.h:363-379). */
typedef struct gd_enepara_raw {
  float vdw[GD_NPT][GD_NLT][2];
  float ele[GD_NELE];
  float pmf[GD_NPT][GD_NLT][2];
  float hpp[GD_NRES];
  float hpl[GD_NLT][2];
  float hdb[GD_NPT][GD_NLT][2];
  float lj[3];
  float el[2];
  float kde;
  float w[GD_NTERM];
  float a_para[GD_NTERM];
  float b_para[GD_NTERM];
} gd_enepara_raw;

/* Kernel-ready force field (EnePara, dock.h:386-421), same field order.
 * Build it with gd_enepara_optimize(). */
typedef struct gd_enepara {
  float p1a[GD_NLT][GD_NPT];
  float p2a[GD_NLT][GD_NPT];
  float lj0, lj1;
  float el0;
  float el1;
  float ele[GD_NELE];
  float a1;
  float b1;
  float pmf0[GD_NLT][GD_NPT];
  float pmf1[GD_NLT][GD_NPT];
  float hdb0[GD_NLT][GD_NPT];
  float hdb1[GD_NLT][GD_NPT];
  float hdb2[GD_NLT][GD_NPT];
  float hpp[GD_NRES];
  float hpl0[GD_NLT];
  float hpl1[GD_NLT];
  float hpl2[GD_NLT];
  float kde2;
  float kde3;
  float w[GD_NTERM];
  float a_para[GD_NTERM];
  float b_para[GD_NTERM];
} gd_enepara;

/* Derives the kernel tables: p1a = 2 eps (s r)^9, p2a = 3 eps (s r)^6,
 * hdb1 = 1/sigma, hpl2 = log(1/(sigma sqrt(2 pi))), kde2 = -1/(2h^2),
 * kde3 = (h sqrt(2 pi))^3.  Replaces OptimizeEnepara (util.C:405-458). */
gd_status gd_enepara_optimize(const gd_enepara_raw *raw, gd_enepara *out);

/* Geometric temperature ladder T_i = T_floor * r^i and minus_beta = -1/T_i
 * (k_B = 1).  n == 1 uses the floor temperature.  Replaces SetTemperature
 * (util.C:491-532).  temps may be NULL. */
gd_status gd_set_temperature(int n_tmp, float floor_temp, float ceiling_temp,
                             float *temps, float *minus_beta);

/* Rigid poses given as [n_pose][7] {tx, ty, tz, qw, qx, qy, qz} (any
 * non-zero quaternion; it is normalised) to the [n_pose][6] move vectors
 * the pose and MC entry points take: the translation, then the ZYX angles
 * (m3, m4, m5) with R = Rz(m3) Ry(m4) Rx(m5) as Move_d builds it
 * (move_d.cu:90-105), m4 in [-pi/2, pi/2].  Host only; no context needed.
 * Zero or non-finite quaternions give GD_EINVAL. */
gd_status gd_poses_from_quaternions(int n_pose, const float *quat_poses, float *poses);

/* ------------------------------------------------------------------------ */
/* Inputs (host, caller-owned).  Structure-of-arrays, no capacity caps.      */
/* ------------------------------------------------------------------------ */

/* Protein: pnp effective points, n_conf conformations.  Point properties are
 * shared by all conformations; coordinates are per conformation.  The fields
 * are those of Protein (dock.h:254-274) after CopyProteinResidue
 * (util.C:253-275). */
typedef struct gd_protein {
  int pnp;
  int n_conf;
  const float *x, *y, *z;      /* [n_conf * pnp]                           */
  const int *t;                /* [pnp] point type, 0..GD_NPT-1            */
  const int *c;                /* [pnp] point class, 0..3                  */
  const float *ele;            /* [pnp] ele[t == 0 ? d + 30 : t]           */
  const int *seq3r;            /* [pnp] residue serial, index into psp row */
  const int *c0_and_d12_or_c2; /* [pnp] (c == 0 && d == 12) || c == 2      */
  const float *hpp;            /* [pnp] hpp[d]                             */
  float pocket_center[3];
} gd_protein;

/* Ligand: lna atoms, n_conf conformations with coordinates relative to the
 * ligand centre (coord_orig of Ligand, dock.h:191-216, after OptimizeLigand
 * util.C:200-226 which sets center := pocket centre). */
typedef struct gd_ligand {
  int lna;
  int n_conf;
  const float *x, *y, *z;      /* [n_conf * lna]                           */
  const int *t;                /* [lna] atom type, 0..GD_NLT-1             */
  const float *c;              /* [lna] partial charge                     */
  const int *n;                /* [lna] atom number; MCS field = n + 1     */
  float center[3];             /* coord_orig.center                        */
} gd_ligand;

/* Pocket-specific potential psp[lig type][seq3r] (Psp, dock.h:289-295). */
typedef struct gd_psp {
  int n_col;                   /* row length; every seq3r must be < n_col  */
  const float *psp;            /* [GD_NLT * n_col]                         */
} gd_psp;

/* KDE points (Kde, dock.h:317-325). */
typedef struct gd_kde {
  int pnk;
  const float *x, *y, *z;      /* [pnk]                                    */
  const int *t;                /* [pnk] ligand atom type                   */
} gd_kde;

/* LHM position restraints (Mcs, dock.h:347-354): pos MCS records of n_field
 * coordinates each; absent atoms hold GD_MCS_INVALID_COORD. */
typedef struct gd_mcs {
  int pos;
  int n_field;                 /* > max(ligand n) + 1; reference MAXMCS=256 */
  const float *x, *y, *z;      /* [pos * n_field]                          */
  const float *tcc;            /* [pos]                                    */
} gd_mcs;

/* One docking complex: a ligand ensemble against a protein ensemble with its
 * pocket template and force field.  The replica grid is protein conformation
 * x temperature x ligand conformation, flat index
 * r = n_tmp * n_lig * p + n_lig * t + l  (SetReplica, util.C:538-558). */
typedef struct gd_complex {
  gd_ligand lig;
  gd_protein prt;
  gd_psp psp;
  gd_kde kde;
  gd_mcs mcs;
  const gd_enepara *ff;
} gd_complex;

/* Checks every size, type code and index of a complex. */
gd_status gd_complex_validate(const gd_complex *cx);

/* ------------------------------------------------------------------------ */
/* Input files (host): the loaders of load.C and the table derivation of     */
/* util.C:200-458 that linear_dock runs before Run.                          */
/* ------------------------------------------------------------------------ */
/* A loaded complex owns its arrays; gd_loaded_complex gives the gd_complex
 * view of them (valid until gd_loaded_free).
 *  pdb:  protein ensemble, MODEL/ENDMDL models; each residue becomes its CA
 *        point, a peptide-plane point and its side-chain points, each the
 *        mean of its atoms per model (loadProtein, load.C:595-990).
 *  sdf:  ligand, one SD record: the atom block gives the default pose, the
 *        OB_ATOM_TYPES / OB_ATOMIC_CHARGES properties types and charges, and
 *        ENSEMBLE_COORDS one conformation per line; conformations within
 *        0.1 A RMSD of the default pose (after optimal superposition) are
 *        dropped, at most 70 are kept (loadLigand, load.C:100-420);
 *        molid is the property tag of the ligand id ("MOLID").
 *  lhm:  pocket template .ff: KDE points, PSP entries and the MCS records
 *        whose ligand id is ligand_id (loadLHM, load.C:1011-1126).
 *  raw:  force field (its ele and hpp tables give the points' ele and hpp,
 *        CopyProteinResidue util.C:253-275).
 *  ff:   the kernel-ready force field the gd_complex view points to.
 * Unreadable files give GD_EIO, malformed content GD_EINVAL. */
typedef struct gd_loaded gd_loaded;
/* The peptide-plane point of a residue (previous residue's C and O, this
 * residue's N) in every model.  Without the flag the points of models after
 * the second are as the reference's loader makes them: from the N atom
 * alone (it looks the previous residue up in a conformation it has not
 * filled yet, load.C:822-833, and finds serial 0 in zeroed memory). */
#define GD_LOAD_PEPTIDE_ALL_MODELS 0x1u
gd_status gd_load(const char *pdb, const char *sdf, const char *lhm,
                  const char *ligand_id, const char *molid,
                  const gd_enepara_raw *raw, const gd_enepara *ff,
                  unsigned flags, gd_loaded **out);
gd_status gd_loaded_complex(const gd_loaded *loaded, gd_complex *out);
/* The ligand id read from the SD record (empty if none). */
const char *gd_loaded_ligand_id(const gd_loaded *loaded);
gd_status gd_loaded_free(gd_loaded *loaded);

/* The force-field parameter files into the raw table, as loadEnePara,
 * loadWeight and loadNorPara (load.C:1139-1419) fill EnePara0:
 *  ff:      tagged lines VDW / PMF / HDB <point> <ligand type> <a> <b>,
 *           ELE <point or residue letter + "C"> <v>, HPP <residue letter>
 *           <v>, HPL <ligand type> <a> <b>, PLJ (3 values), PEL (2), WEI
 *           (up to 10 weights), KDE (bandwidth); other lines are skipped,
 *           missing values read as 0, and the residue hydrophobicities are
 *           rescaled to [-1, 1] afterwards.
 *  weights, nor_a, nor_b: one value per line (first 30 characters) for the
 *           term weights w and the normalisation a_para / b_para, the first
 *           GD_NTERM lines; NULL keeps w from the WEI line and a_para /
 *           b_para at 0.
 * Every entry no line sets is 0.  Unreadable files give GD_EIO; unknown
 * point, ligand or residue names give GD_EINVAL (the reference exits or
 * indexes past its tables).  *out is written only on success. */
gd_status gd_load_enepara(const char *ff, const char *weights, const char *nor_a,
                          const char *nor_b, gd_enepara_raw *out);

/* ------------------------------------------------------------------------ */
/* Device context and device-resident complexes                             */
/* ------------------------------------------------------------------------ */
typedef struct gd_ctx gd_ctx;
typedef struct gd_dcomplex gd_dcomplex;

/* Binds a CUDA device and a stream (NULL = a stream owned by the context;
 * otherwise a cudaStream_t created by the caller on that device). */
gd_status gd_ctx_create(int device, void *stream, gd_ctx **out);
gd_status gd_ctx_destroy(gd_ctx *ctx);
gd_status gd_ctx_sync(gd_ctx *ctx);
/* Number of this library's kernels launched through ctx so far. */
uint64_t gd_ctx_launch_count(const gd_ctx *ctx);

/* Copies a complex to the device in the kernel layout (points packed into
 * 16 B + 8 B records, type-pair table, KDE bucketed by type, MCS gathered per
 * ligand atom).  Replaces the table staging of run.cu:114-256. */
gd_status gd_complex_upload(gd_ctx *ctx, const gd_complex *cx,
                            gd_dcomplex **out);
/* Like gd_complex_upload, but the protein arrays are not copied: the new
 * complex reads conformations [prt_conf0, prt_conf0 + n_prt) of `protein`
 * (an uploaded complex of the same protein, kept alive by the new handle).
 * Used to batch many ligands against one resident protein. */
gd_status gd_complex_upload_shared(gd_ctx *ctx, const gd_complex *cx,
                                   const gd_dcomplex *protein, int prt_conf0,
                                   int n_prt, gd_dcomplex **out);
gd_status gd_complex_free(gd_dcomplex *dcx);
/* Device bytes held by an uploaded complex. */
size_t gd_complex_device_bytes(const gd_dcomplex *dcx);

/* ------------------------------------------------------------------------ */
/* Launch shape of the energy kernel and its autotuner                      */
/* ------------------------------------------------------------------------ */
/* The compute warps of a CTA form an atom_groups x tile_groups grid; each
 * warp keeps atoms_per_warp ligand atoms in registers and sweeps every
 * tile_groups-th protein tile. */
typedef struct gd_tile {
  int atom_groups;
  int tile_groups;
  int atoms_per_warp;
} gd_tile;

/* Times every compiled launch shape for this complex's size class on the
 * REMC kernel (a temporary batch of copies of the complex, one CTA per SM or
 * more, a few MC steps per sample), keeps the fastest in the context and
 * returns it with its time for 4 MC steps; later launches of that size class
 * use it.  Synchronous; takes about a second.  A size class is (ligand-size bucket,
 * protein tiles): ligand sizes are rounded up to a multiple of 8 atoms and a
 * class's shape covers the bucket's largest size, so the ligands of a batch
 * that fall in one bucket share one launch shape. */
gd_status gd_autotune(gd_ctx *ctx, const gd_dcomplex *dcx, gd_tile *best,
                      double *best_ms);
/* Sets the launch shape of a size class explicitly (it must cover the
 * bucket of lna, i.e. lna rounded up to a multiple of 8). */
gd_status gd_ctx_set_tile(gd_ctx *ctx, int lna, int pnp, const gd_tile *tile);

/* How MC launches are spread over the SMs.  A unit is one CTA's worth of
 * replicas (32 lanes).  GD_SCHED_AUTO (the default): a launch with more units
 * than CTAs resident at once runs persistent CTAs, each taking a list of
 * units and step ranges cut so that every CTA does the same amount of work
 * (a unit may run its first steps on one CTA and the rest on another, after
 * a bounded wait); otherwise one CTA per unit.  GD_SCHED_WAVES: always one
 * CTA per unit.  GD_SCHED_PERSISTENT: always the persistent schedule, over
 * `machines` CTAs (0: SMs x resident CTAs per SM).  Trajectories are
 * bit-identical under every schedule.  Applies to launches enqueued after
 * the call (a REMC run or batch keeps the schedule its captured graph was
 * built with). */
enum { GD_SCHED_AUTO = 0, GD_SCHED_WAVES = 1, GD_SCHED_PERSISTENT = 2 };
gd_status gd_ctx_set_schedule(gd_ctx *ctx, int mode, int machines);
/* Persistent launches of a run with one launch shape: the last `tail` MC
 * steps of every unit (default 2; 0: none) are not dealt to the CTAs in
 * advance but left in a queue, one step per piece, that CTAs which have run
 * their own share take from in order, once every CTA of the launch has
 * started.  The CTAs then end within about one unit-step of each other even
 * when units or SMs run at different speeds (contacts, clocks).  Trajectories
 * stay bit-identical.  Applies to runs whose schedule is made after the call;
 * tail is 0..64. */
gd_status gd_ctx_set_schedule_tail(gd_ctx *ctx, int tail);

/* How many CTAs share each 32-replica unit of an MC launch.  With split > 1
 * the unit runs on a thread-block cluster of `split` CTAs (SMs of one GPC):
 * CTA r evaluates the protein tiles r, r + split, ..., the CTAs add their
 * partial energies through distributed shared memory every MC step (in
 * rank order) and all take the same decision.  A complex's run then takes
 * about 1/split of the time when SMs are free (latency), at a few percent
 * more total work.  split = 0 (the default) chooses per complex from its
 * size and its own run: the largest power of two <= ligand-size bucket x
 * protein points / c and <= SMs / units of the run, at most 8, with
 * c = 4,500 for runs and batches (they have the GPU to themselves: a
 * 24-atom ligand against 1,500 points runs on 8 CTAs, an ensemble or batch
 * with more units than SMs unsplit) and c = 42,500 for server requests
 * (each a run of its own among others, so that splitting under load costs
 * little throughput: 120 atoms against 10,000 points on 8 CTAs, 30 atoms
 * against 4,000 on 2); 1, 2, 4 or 8 fix it for every complex.  A run's
 * results depend on its split (the partial sums are added in another
 * order) but never on what runs beside it.  Applies to runs, batches and
 * server lanes created after the call. */
gd_status gd_ctx_set_split(gd_ctx *ctx, int split);

/* ------------------------------------------------------------------------ */
/* Pose energies (CalcEnergy_d after Move_d on a given move vector)         */
/* ------------------------------------------------------------------------ */
/* A pose is a 6-float move vector (tx, ty, tz, rx, ry, rz), the reference's
 * movematrix: x = R_zyx(rx, ry, rz) * x_orig + t + centre (move_d.cu:86-127).
 * terms: [n_pose][GD_NTERM] normalised terms + weighted total (FP32).
 * raw:   [n_pose][GD_NRAW] un-normalised terms in FP64 (may be NULL).
 * The _dev form takes device pointers and runs on the context stream without
 * synchronising; the host form copies poses in and results out. */
gd_status gd_energy_poses_dev(gd_ctx *ctx, const gd_dcomplex *dcx,
                              int prt_conf, int lig_conf, int n_pose,
                              const float *poses_dev, float *terms_dev,
                              double *raw_dev);
gd_status gd_energy_poses(gd_ctx *ctx, const gd_dcomplex *dcx, int prt_conf,
                          int lig_conf, int n_pose, const float *poses,
                          float *terms, double *raw);

/* Same computation and results as gd_energy_poses (host buffers), without
 * allocating any device memory. It has no counterpart in the reference.
 *
 * Who needs it: a caller that has handed its spare device memory to another
 * allocator (the serving form's HBM budget, a framework's caching
 * allocator) can see even a small cudaMalloc/cudaMallocAsync fail, and a
 * caller may want no allocator call at all on its scoring path. This entry
 * point stages poses, results and the launch descriptor in one fixed
 * device array compiled into the library (about 2.2 MB per device) instead.
 *
 * Limit: n_pose <= GD_NOALLOC_MAX_POSES; larger calls return GD_EINVAL
 * before anything runs (split them, or use gd_energy_poses).  An empty call
 * (n_pose == 0) returns GD_OK whatever the other arguments, as
 * gd_energy_poses does.
 * Set-up: the array is committed on the device, and its address in the
 * current CUDA context looked up, by gd_ctx_create (CUDA loads the module
 * that holds it lazily; doing it there keeps the allocation out of this
 * entry point).  So the calls themselves allocate nothing, and the memory
 * the array needs is taken when the context is created.  A gd_ctx must not
 * outlive the CUDA context it was created in: after cudaDeviceReset, create
 * a new gd_ctx.
 * Nothing in the array has to start at zero: each call writes what the kernel
 * reads before the launch.
 * Overlapping calls race: there is one array per device, shared by every
 * context and thread of the process, and calls are not serialised. Do not
 * let two calls on the same device run at the same time. Each call waits
 * for its own results before it returns. */
#define GD_NOALLOC_MAX_POSES 16384
gd_status gd_energy_poses_noalloc(gd_ctx *ctx, const gd_dcomplex *dcx,
                                  int prt_conf, int lig_conf, int n_pose,
                                  const float *poses, float *terms,
                                  double *raw);

/* Contact-mode similarity matrix of trajectory conformations
 * (SimilarityMatirxGen CalculateSimilarityMatrix, util.C:37-193).
 * confs[n_conf][8] are the rows of a trace file: protein conformation and
 * ligand conformation (as floats, truncated to int), then the move vector
 * (6).  similarity[n_conf][n_conf] (host) gets, at (i, j), the Matthews
 * correlation of conformation j's contacts (ligand atom / protein point with
 * dst <= pmf0) against conformation i's contact map, or GD_CMCC_INVALID
 * where it is undefined, computed with the reference's float arithmetic:
 * identical to the reference's values.  Conformations out of the complex's
 * range, or non-finite values, give GD_EINVAL.  Device memory: about
 * n_conf * (4 n_conf + lna * pnp / 8) bytes, freed before returning. */
gd_status gd_similarity_matrix(gd_ctx *ctx, const gd_dcomplex *dcx, int n_conf,
                               const float *confs, float *similarity);
/* The same matrix written to device memory of the context's device
 * (similarity_dev: n_conf * n_conf floats), for callers that keep it on the
 * GPU; confs stay host memory.  Returns when the matrix is complete. */
gd_status gd_similarity_matrix_dev(gd_ctx *ctx, const gd_dcomplex *dcx, int n_conf,
                                   const float *confs, float *similarity_dev);

/* ------------------------------------------------------------------------ */
/* Replica-exchange Monte Carlo                                             */
/* ------------------------------------------------------------------------ */
#define GD_MC_EXCHANGE   0x1u  /* temperature exchange (IS_EXCHANGE)        */
#define GD_MC_MOVE_AWAY  0x2u  /* initial MoveAway_d + forced accept        */
#define GD_MC_RECORD     0x4u  /* per-step trajectory record (IS_OUTPUT)    */
/* Contact-map Matthews correlation of every pose (IS_CALCU_MCC,
 * calcmcc_d.cu:57-213): contacts are ligand-atom / protein-point pairs with
 * d <= pmf0; the reference map is that of ligand conformation 0 in its start
 * pose against the complex's first protein conformation.  Per step
 * cmcc = (tp tn - fp fn) / sqrt((tp+fp)(tp+fn)(tn+fp)(tn+fn)), or 10000 when
 * the denominator is 0.  It follows the accepted state and is reported in
 * gd_record.cmcc; it never enters the acceptance. */
#define GD_MC_MCC        0x8u
#define GD_CMCC_INVALID  10000.0f
/* Bayesian total (IS_BAYE, calcenergy_d.cu:311-347): e[GD_E_TOTAL] =
 * sum of log10 densities of the nine normalised terms under the low-decoy
 * distributions minus the same under the high-decoy distributions
 * (families and parameters of util_d.cu:220-290 and distribution.h), in
 * place of the weighted sum.  It is the energy the Metropolis test and the
 * exchange use. */
#define GD_MC_BAYES      0x10u

typedef struct gd_mc_params {
  int steps_total;           /* MC steps per replica                        */
  int steps_per_exchange;    /* MC steps between exchanges                  */
  int steps_per_dump;        /* the exchange parity restarts every dump     */
                             /* (gpusingle.cu:14-18); <= 0 means never      */
  int n_tmp;                 /* temperatures per (prt, lig) group           */
  float move_scale[6];       /* translation x y z, rotation x y z           */
  const float *minus_beta;   /* [n_tmp] -1/T per temperature index          */
  uint64_t seed;             /* Philox4x32-10 key                           */
  uint32_t stream_id;        /* second key word (request id when serving)   */
  uint32_t flags;            /* GD_MC_*                                     */
} gd_mc_params;

/* Per-step trajectory record: the fields of LigRecordSingleStep
 * (dock.h:487-493), i.e. the accepted state at the start of each step, plus
 * the proposed total energy of that step and the Metropolis decision, so a
 * run can be replayed decision by decision. */
typedef struct gd_record {
  int idx_rep, idx_prt, idx_tmp, idx_lig;
  float e[GD_NTERM];
  float cmcc;
  float movematrix[6];
  int step;
  float e_prop_total;
  int accepted;
} gd_record;

/* Results, the fields of McLog (dock.h:472-482) plus the final state.  Every
 * pointer may be NULL; sizes are those of the run. */
typedef struct gd_mc_log {
  double t_compute;          /* seconds of device time in MC + exchange     */
  double t_wall;             /* seconds including copies                    */
  int64_t ac_mc;             /* accepted MC moves, all replicas             */
  int64_t ac_temp_exchg;     /* accepted exchanges (2 per swap)             */
  int *acs_mc;               /* [n_rep]                                     */
  int *acs_temp_exchg;       /* [n_tmp] counted by slot t as                */
                             /* exchangereplicas_d.cu:63-64 does            */
  float *energy;             /* [n_rep][GD_NTERM] accepted energy           */
  float *movematrix;         /* [n_rep][6] accepted move vector             */
  int *idx_tmp;              /* [n_rep] temperature index of each replica   */
  gd_record *record;         /* [n_rep][steps_total] with GD_MC_RECORD      */
} gd_mc_log;

typedef struct gd_remc gd_remc;

gd_status gd_remc_create(gd_ctx *ctx, const gd_dcomplex *dcx,
                         const gd_mc_params *mc, gd_remc **out);
/* MonteCarlo_Init_d (montecarlo_d.cu:12-55): optional move-away with forced
 * accept, initial energies, counters zeroed, step counter reset. */
gd_status gd_remc_init(gd_remc *remc);
/* Runs n_steps MC steps of every replica with an exchange after every
 * steps_per_exchange steps (n_steps must be a multiple of it). Asynchronous. */
gd_status gd_remc_run(gd_remc *remc, int n_steps);
gd_status gd_remc_read(gd_remc *remc, gd_mc_log *log);
gd_status gd_remc_destroy(gd_remc *remc);
/* Trajectory files, the IS_OUTPUT dumps of gpusingle.cu:24-32.  After the
 * call, every completed dump of mc.steps_per_dump MC steps (a multiple of
 * steps_per_exchange) is written to {dir}/{stem}_NNNN.bin (NNNN = 0000,
 * 0001, ...): n_rep LigRecord of steps_per_dump LigRecordSingleStep
 * (dock.h:487-501; gd_record's first 88 bytes), replica-major, the bytes
 * DumpLigRecord (hdf5io.C:11-32) stores in dataset "dset".
 * {dir}/{stem}.layout.json describes that layout (field names, offsets and
 * types, for a numpy structured dtype or an HDF5 compound type).  The
 * kernel writes the records into a two-dump device ring; each completed dump
 * is copied to pinned host memory on a side stream while the next one runs,
 * and written from there, so the MC steps do not wait for the disk.  Steps
 * of an unfinished dump are not written.  The in-memory record
 * (gd_mc_log.record) is not filled while a trajectory is set.  Call before
 * gd_remc_init; writing errors surface as GD_EIO from gd_remc_run /
 * gd_remc_read. */
gd_status gd_remc_set_trajectory(gd_remc *remc, const char *dir,
                                 const char *stem);
/* Checkpoint / resume (no counterpart in the reference, which keeps no
 * random-number state in its dumps, util_d.cu:85-92, and cannot resume).
 * gd_remc_snapshot writes the run's state into host memory: a header naming
 * the run's shape (replicas, temperatures, ligand and protein sizes, seed,
 * stream id, flags) and step counter, then every replica's accepted move
 * vector, energy, MCC, temperature index and acceptance counter and the
 * exchange counters per temperature slot.  With buf == NULL it only sets
 * *size; otherwise cap must be at least *size.  It waits for the run's
 * enqueued work and fails with that work's error, if any.
 * gd_remc_restore loads such a snapshot into a run created with the same
 * complex sizes and MC parameters (GD_EINVAL otherwise) and sets its step
 * counter; the next gd_remc_run continues from there.  The random stream is
 * counter-based (key: seed, stream id; counter: replica, step), so a run
 * snapshotted at step s and restored into a new handle gives the same
 * trajectory, bit for bit, as one run without the break.  The in-memory
 * record (GD_MC_RECORD) of steps before s is not part of a snapshot. */
gd_status gd_remc_snapshot(gd_remc *remc, void *buf, size_t cap, size_t *size);
gd_status gd_remc_restore(gd_remc *remc, const void *buf, size_t size);
int gd_remc_n_rep(const gd_remc *remc);
/* CUDA-event timing of the MC kernels and exchange kernels issued by
 * gd_remc_run / gd_batch_run while profiling is on.  One MC sample spans the
 * launches of all launch shapes of one interval (they run side by side on
 * side streams), so with a single shape it is one kernel's duration.
 * gd_remc_kernel_times synchronises, returns the sums and sample counts
 * since the previous call and resets them. */
gd_status gd_remc_set_profiling(gd_remc *remc, int on);
gd_status gd_remc_kernel_times(gd_remc *remc, double *mc_ms, int *mc_launches,
                               double *exch_ms, int *exch_launches);

/* One call with host buffers: upload, init, steps_total steps, read back,
 * free.  The counterpart of Run (run.cu:41-353).  Runs on device 0 through a
 * context that each calling thread creates on its first call and keeps
 * (stream, side streams, launch-shape cache); nothing of a run outlives the
 * call. */
gd_status gd_run(const gd_complex *cx, const gd_mc_params *mc,
                 gd_mc_log *log);

/* ------------------------------------------------------------------------ */
/* Batched form: many complexes of uneven sizes advanced together.  All     */
/* share steps_per_exchange; each keeps its own replicas, temperatures,     */
/* random stream and counters.  Complexes with the same launch shape share  */
/* one launch; with whole exchange groups per CTA (32 % n_tmp == 0) the     */
/* exchange runs inside the kernel and a run is one launch per shape (side  */
/* by side), replayed from one captured CUDA graph once a run length is     */
/* used again; otherwise the interval sequence is replayed from a captured  */
/* CUDA graph.                                                              */
/* ------------------------------------------------------------------------ */
typedef struct gd_batch gd_batch;

gd_status gd_batch_create(gd_ctx *ctx, int n, const gd_dcomplex *const *items,
                          const gd_mc_params *params, gd_batch **out);
gd_status gd_batch_init(gd_batch *batch);
gd_status gd_batch_run(gd_batch *batch, int n_steps);
/* Results of complex `item` (same layout as gd_remc_read). */
gd_status gd_batch_read(gd_batch *batch, int item, gd_mc_log *log);
gd_status gd_batch_destroy(gd_batch *batch);
int gd_batch_n_rep(const gd_batch *batch);
int gd_batch_n_launch_shapes(const gd_batch *batch);
/* Checkpoint / resume of a whole batch, as gd_remc_snapshot / restore. */
gd_status gd_batch_snapshot(gd_batch *batch, void *buf, size_t cap, size_t *size);
gd_status gd_batch_restore(gd_batch *batch, const void *buf, size_t size);
gd_status gd_batch_set_profiling(gd_batch *batch, int on);
gd_status gd_batch_kernel_times(gd_batch *batch, double *mc_ms, int *mc_launches,
                                double *exch_ms, int *exch_launches);

/* ------------------------------------------------------------------------ */
/* Serving form: a request loop with continuous batching.  Proteins are     */
/* uploaded once and stay resident; requests (a ligand ensemble + pocket    */
/* template + MC parameters against a resident protein) are copied at       */
/* submit, admitted by a scheduler thread while the HBM budget and the      */
/* slot count allow, and advanced together in iterations, each with its own */
/* step counter, state and random stream, so a request's result does not    */
/* depend on what else is running.  In an iteration the most expensive      */
/* active request (ligand atoms x protein points) advances steps_per_launch */
/* MC steps (at least one exchange interval) and cheaper ones               */
/* proportionally more, in whole exchange intervals, so that no request     */
/* holds the others back.  Short iterations keep the SMs busier: on the     */
/* serving trace (10-step exchange interval) 20 steps per launch served     */
/* 63.8 req/s at SM occupancy 0.86, against 60.2 / 0.81 with 100 and        */
/* 54.8 / 0.74 with 400.                                                    */
/* ------------------------------------------------------------------------ */
typedef struct gd_server gd_server;

typedef struct gd_server_stats {
  int queued;               /* waiting for admission                        */
  int active;               /* admitted, running                            */
  uint64_t completed;       /* finished successfully                        */
  uint64_t iterations;      /* scheduler iterations                         */
  uint64_t launches;        /* kernel launches issued                       */
  size_t bytes_in_use;      /* device bytes held (proteins + requests)      */
  double busy_s;            /* seconds the scheduler spent in iterations    */
  double cta_busy_s;        /* seconds the server's CTAs spent on SMs,      */
                            /* summed over CTAs (/ SMs / wall = occupancy)  */
  double host_launch_s;     /* scheduler-thread time spent issuing launches */
} gd_server_stats;

/* max_active <= 0 means two requests per SM. */
gd_status gd_server_create(int device, size_t hbm_budget_bytes, int max_active,
                           int steps_per_launch, gd_server **out);
/* Makes the protein (all conformations) of cx resident; returns its id. */
gd_status gd_server_add_protein(gd_server *srv, const gd_complex *cx, int *protein_id);
/* Copies the request (cx->prt is ignored: the resident protein is used).
 * GD_EBUDGET when it can never fit the budget.  With GD_MC_RECORD in
 * mc->flags the request also keeps its per-step record on the device
 * (n_rep x steps_total gd_record, counted in its budget), returned through
 * log->record by gd_server_poll / gd_server_wait. */
gd_status gd_server_submit(gd_server *srv, int protein_id, const gd_complex *cx,
                           const gd_mc_params *mc, uint64_t *req_id);
/* GD_EAGAIN while queued or running; GD_OK with the results (t_wall = latency
 * from submit, t_compute = time since admission) and the request released;
 * GD_ECANCELLED / the failure status otherwise. */
gd_status gd_server_poll(gd_server *srv, uint64_t req_id, gd_mc_log *log);
/* As poll, blocking up to timeout_ms (GD_ETIMEDOUT after). */
gd_status gd_server_wait(gd_server *srv, uint64_t req_id, int timeout_ms,
                         gd_mc_log *log);
gd_status gd_server_cancel(gd_server *srv, uint64_t req_id);
gd_status gd_server_get_stats(gd_server *srv, gd_server_stats *out);
/* The server's own context (owned by the server; do not destroy it).  Its
 * launch shapes (gd_autotune, gd_ctx_set_tile) and split rule
 * (gd_ctx_set_split) apply to requests admitted after the call. */
gd_ctx *gd_server_context(gd_server *srv);
gd_status gd_server_destroy(gd_server *srv);

/* ------------------------------------------------------------------------ */
/* Building blocks exposed for testing: the Metropolis and exchange rules   */
/* on given energies, the counter-based RNG and the decision exp.           */
/* ------------------------------------------------------------------------ */
/* accept[i] = u(seed, stream, rep[i], step[i]) < gd_expf(dE[i] * mbeta[i]) */
gd_status gd_metropolis_dev(gd_ctx *ctx, int n, const float *e_new,
                            const float *e_old, const float *minus_beta,
                            const int *rep, const int *step, uint64_t seed,
                            uint32_t stream_id, int *accept);
/* Philox4x32-10 blocks and exp evaluated on the device (device pointers). */
gd_status gd_philox_dev(gd_ctx *ctx, int n, const uint32_t *ctr4,
                        const uint32_t *key2, uint32_t *out4);
gd_status gd_expf_dev(gd_ctx *ctx, int n, const float *x, float *y);
/* FP32 FMA throughput probe (roofline denominator): n_blocks x 256 threads,
 * 8 chains x 16 FMAs x iters each; returns the time and the flop count. */
gd_status gd_fma_peak(gd_ctx *ctx, int n_blocks, int iters, float *ms,
                      double *flops);
/* Test hook for the failure path of the persistent schedule's bounded
 * waits (a CTA that continues a unit waits for the CTA that ran the unit's
 * earlier steps).  MC launches enqueued through ctx after the call give up
 * such a wait after wait_limit polls of about 256 ns each (0: the default,
 * 2^24 polls, about 4 s).  With never_release != 0 every such wait targets
 * a step no run reaches, so each one runs out after wait_limit polls: the
 * kernel records the error and finishes, and the next call that checks the
 * context's error word (gd_remc_read, gd_ctx_sync, ...) returns
 * GD_ETIMEDOUT and clears it.  The results of such a run are undefined.
 * never_release needs a nonzero wait_limit.  gd_ctx_set_wait_test(ctx, 0, 0)
 * restores the defaults (runs created meanwhile keep the setting their
 * captured launches were built with). */
gd_status gd_ctx_set_wait_test(gd_ctx *ctx, unsigned wait_limit, int never_release);
/* Test hook for allocation failures: the nth device allocation the library
 * makes through ctx from now on (uploads, run state, server requests; nth
 * >= 1) fails as cudaMallocAsync does on a full device, and the call that
 * made it returns GD_ENOMEM after freeing what it had allocated.  The hook
 * is then off again; nth = 0 turns it off. */
gd_status gd_ctx_set_alloc_fail(gd_ctx *ctx, int nth);
/* The persistent schedule (host only, no device): n_units units of cost[u]
 * per MC step and steps[u] steps over `machines` CTAs.  pieces[4 k ..] =
 * {unit, first step, end step, wait} for k < piece_off[*n_used], CTA m's in
 * piece_off[m] .. piece_off[m+1]-1 in run order; cap = room in pieces (in
 * pieces of 4 ints), piece_off holds machines + 1 ints. */
gd_status gd_schedule_pieces(const double *cost, const int *steps, int n_units,
                             int machines, int *pieces, int cap, int *piece_off,
                             int *n_used);
/* The persistent schedule with a shared queue (host only): the first
 * steps[u] - tail steps of every unit cut as by gd_schedule_pieces over
 * `machines` CTAs (piece_off: machines + 1 entries), followed by *n_queue
 * one-step pieces {unit, step, step + 1, wait} (the last `tail` steps of every
 * unit, step by step, units in the order their first part ends). */
gd_status gd_schedule_queue(const double *cost, const int *steps, int n_units, int machines,
                            int tail, int *pieces, int cap, int *piece_off, int *n_queue);

#ifdef __cplusplus
}
#endif
#endif /* GPUDOCK_H */
