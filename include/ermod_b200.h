/*
 * ermod_b200.h -- C-ABI of the B200 (sm_100a) energy-distribution engine.
 *
 * This library replaces the per-frame hot path of ERmod's `erdst`:
 *   realcal   (erdst/realcal.F90)   solute-solvent LJ + real-space Ewald pair energies
 *   insertion (erdst/insertion.F90) test-particle placement for refs mode
 *   recpcal   (erdst/recpcal.F90)   smooth-PME reciprocal-space energies (cuFFT for the FFT)
 *   engproc   (erdst/engproc.F90)   binning onto the energy mesh, edens / ecorr accumulation
 *
 * The reference drives that path through the module-procedure trio
 *   engclear        erdst/engproc.F90:321-340
 *   engconst(stnum) erdst/engproc.F90:353-517
 *   engstore(stnum) erdst/engproc.F90:520-725
 * called from trjmain (erdst/enganal.F90:86-95) with all state in module
 * `engmain` (erdst/engmain.F90:314-348).  The entry points below keep that
 * call structure: a Fortran host binds them through ISO_C_BINDING
 * (bind(C) interfaces over these plain-C signatures), a C/C++ host calls
 * them directly.  All state lives in an opaque context instead of module globals.
 *
 * Conventions
 *   - Plain C types only.  Arrays are caller-owned HOST memory unless a
 *     name ends in `_dev`.  Multi-dimensional arrays use the reference's
 *     Fortran (column-major) layout: sitepos(3, n) is x,y,z per atom.
 *   - Indices stored in arrays (ljtype, uvspec, ...) are 1-based as in the
 *     reference.
 *   - Every call is synchronous: on return the device work is complete and
 *     host outputs are written.
 *   - Return value: 0 success, > 0 warning (the reference's `warning`,
 *     erdst/mpiproc.F90:238-252), < 0 error (the reference's
 *     `halt_with_error`, erdst/mpiproc.F90:181-236).  The reference's
 *     7-character code ("eng_min", "eng_sft", ...) is available from
 *     ermod_last_error().  The library never aborts the process.
 *   - One context per host thread; a context is not re-entrant.
 */
#ifndef ERMOD_B200_H
#define ERMOD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ERMOD_ABI_VERSION 3

/* ---- status codes --------------------------------------------------- */
#define ERMOD_OK               0
#define ERMOD_WARN_MBIN        1   /* warning('mbin'): energy in the last bin (engproc.F90:1161-1166) */
#define ERMOD_ERR_ARG        (-1)  /* invalid argument / unsupported parameter combination */
#define ERMOD_ERR_CUDA       (-2)  /* CUDA / cuFFT failure */
#define ERMOD_ERR_ENG_MIN   (-10)  /* halt_with_error('eng_min') engproc.F90:1143-1146 */
#define ERMOD_ERR_ENG_SFT   (-11)  /* halt_with_error('eng_sft') engproc.F90:1151-1156 */
#define ERMOD_ERR_ENG_CNS   (-12)  /* halt_with_error('eng_cns') engproc.F90:924 */
#define ERMOD_ERR_RCP_CNS   (-13)  /* halt_with_error('rcp_cns') recpcal.F90:350 */
#define ERMOD_ERR_INS_GEO   (-14)  /* halt_with_error('ins_geo') insertion.F90:154-156 */
#define ERMOD_ERR_ENG_ECD   (-15)  /* halt_with_error('eng_ecd') engproc.F90:193 (mesh) */
#define ERMOD_ERR_CELL      (-16)  /* cell too small for the cutoff (realcal.F90:849-856) */
#define ERMOD_ERR_OVERFLOW  (-17)  /* an internal fixed-size limit was exceeded */
#define ERMOD_ERR_UNSUPPORTED (-20)

/* ---- constants mirrored from erdst/engmain.F90:352-375 --------------- */
#define ERMOD_SLT_SOLN        1
#define ERMOD_SLT_REFS_RIGID  2
#define ERMOD_SLT_REFS_FLEX   3
#define ERMOD_PT_SOLVENT      0
#define ERMOD_PT_SOLUTE       1
#define ERMOD_PT_TEST_RIGID   2
#define ERMOD_PT_TEST_FLEX    3
#define ERMOD_SYS_NONPERIODIC 0
#define ERMOD_SYS_PERIODIC    1
#define ERMOD_ES_NVT          1
#define ERMOD_ES_NPT          2
#define ERMOD_EL_COULOMB      0
#define ERMOD_EL_EWALD        1
#define ERMOD_EL_PME          2
#define ERMOD_EL_PPPM         3
#define ERMOD_LJSWT_POT_CHM   0
#define ERMOD_LJSWT_POT_GMX   1
#define ERMOD_LJSWT_FRC_CHM   2
#define ERMOD_LJSWT_FRC_GMX   3
#define ERMOD_INSPOS_RANDOM   0
#define ERMOD_INSPOS_NOCHANGE 1
#define ERMOD_INSPOS_SPHERE   2   /* COM at the host aggregate centre + a point of the shell lwreg..upreg */
#define ERMOD_INSPOS_SLAB_GENERIC   3   /* + cell . (u1, u2, dz / |c3|), lwreg < dz < upreg */
#define ERMOD_INSPOS_SLAB_SYMMETRIC 4   /* the same with dz of either sign */
#define ERMOD_INSPOS_RMSD     5   /* translation within upreg + 3 r_max of the fitted reference, RMSD lwreg..upreg */
#define ERMOD_INSPOS_GAUSS    6   /* uniform / Gaussian mixture around the fitted reference (experimental) */
/* insposition 5 and 6 (insorigin 3) need ermod_set_refstructure before the first frame */
#define ERMOD_INSSTR_NOREJECT 0   /* insstructure (engmain.F90) */
#define ERMOD_INSSTR_RMSD     1
#define ERMOD_INSROT_RANDOM   0
#define ERMOD_INSROT_NOCHANGE 1

/* Insertion proposal (refs mode). */
#define ERMOD_PROPOSAL_UNIFORM 0   /* the reference's uniform insertion (insertion.F90:152-162) */
#define ERMOD_PROPOSAL_LEARNED 1   /* MLP voxel proposal mixed with uniform, p/q weighted */

/*
 * Run parameters: &ene_param after iniparam (erdst/setconf.F90:133-438)
 * has applied its defaults.  `temp` is kcal/mol (setconf.F90:304).
 * cltype: ERMOD_EL_COULOMB, ERMOD_EL_PME, or ERMOD_EL_PPPM with an even splodr
 * (recpcal_pppm_greenfunc, recpcal.F90:217-337); ERMOD_EL_EWALD is refused
 * ("set_prs") as setconf.F90:318-320 refuses it.
 */
typedef struct ermod_params {
  int32_t slttype, boxshp, estype, cltype, ljswitch;
  int32_t splodr, ms1max, ms2max, ms3max;
  int32_t maxins;                 /* insertions per frame (refs); ignored in soln */
  int32_t corrcal, selfcal, wgtslf;
  int32_t insposition, insorient;
  int32_t iseed;                  /* seed of the insertion random stream */
  double  temp;                   /* kcal/mol */
  float   elecut, lwljcut, upljcut, screen;
  /* engine options (no reference counterpart; 0 = automatic) */
  int32_t ins_chunk;              /* insertions per PME chunk: 0 or 32 (the chunk is one warp lane per
                                     insertion; other values are refused with "ins_chk") */
  int32_t ecorr_batch;            /* insertions per ecorr GEMM batch (0 = auto) */
  int32_t weight_bits;            /* fixed-point bits of ecorr weights (0 = 24) */
  int32_t proposal;               /* ERMOD_PROPOSAL_* */
  int32_t keep_uvengy;            /* 1: keep per-molecule energies for ermod_get_uvengy */
  int32_t ecorr_path;             /* 0: INT8 tensor-core GEMM, 1: FP64 CUDA-core kernel */
  int32_t spectrum_path;          /* PME solve. 0: automatic, 1: spread grid + cuFFT R2C/C2R,
                                     2: fused solve, spectrum by direct site sums,
                                     3: fused solve, spectrum by plane spreading + FFT
                                     (2 and 3 need power-of-two meshes of 16..128) */
  int32_t graph_mode;             /* 0: a frame runs as one CUDA graph launch (captured again
                                     only when the frame's constants change), 1: direct launches */
  int32_t stage_timing;           /* 1: CUDA events between stages for ermod_get_timings
                                     (implies direct launches); 0: total frame time only */
  /* insertion region, insposition 2..4 (&ene_param lwreg, upreg, hostspec; engmain.F90:55-58, 77-90, 126-127).
     The solute COM is first moved to the mass-weighted centre of the host aggregate (insorigin 2,
     com_aggregate insertion.F90:587-614), then shifted as insertion.F90:164-200 does. */
  float   lwreg, upreg;
  int32_t hostspec;               /* bit (sp - 1) set: solvent species sp (uvspec) belongs to the host */
  /* structure check of solutes in solution (&ene_param insstructure, lwstr, upstr): with
     ERMOD_INSSTR_RMSD a solute whose best-fit RMSD from RefInfo's solute lies outside
     [lwstr, upstr] is skipped for the frame (check_mol_configuration, engproc.F90:1277-1295).
     Refs mode ignores these: getsolute's filter acts on the conformations the host passes. */
  int32_t insstructure;
  float   lwstr, upstr;
} ermod_params;

/*
 * System topology after setparam (erdst/setconf.F90:516-844).
 * Molecules are ordered as in the reference: for refs mode the test
 * particle is the LAST molecule (engproc.F90:99-101).  Atom arrays cover
 * numatm = sum(numsite) atoms, i.e. one copy of the test particle.
 */
typedef struct ermod_topology {
  int32_t nummol;
  const int32_t* numsite;     /* [nummol] */
  const int32_t* sluvid;      /* [nummol] ERMOD_PT_* */
  const int32_t* uvspec;      /* [nummol] solvent species 1..numslv, 0 = solute (engproc.F90:112-118) */
  const float*   charge;      /* [numatm] already x18.22261721 (setconf.F90:834) */
  const int32_t* ljtype;      /* [numatm] 1-based into the LJ tables */
  const float*   sitemass;    /* [numatm] */
  int32_t        ljtype_max;
  const float*   ljene_mat;   /* [ljtype_max*ljtype_max] column-major (setconf.F90:813-826) */
  const float*   ljlensq_mat; /* [ljtype_max*ljtype_max] */
  const float*   bfcoord;     /* [3*s] body-fixed test-particle coordinates (refs rigid), else NULL */
} ermod_topology;

/* Energy mesh built by enginit (erdst/engproc.F90:36-319). */
typedef struct ermod_mesh {
  int32_t numslv, ermax, esmax;
  const double*  uvcrd;      /* [ermax] concatenated over species */
  const int32_t* uvmax;      /* [numslv] */
  const int32_t* uvsoft;     /* [numslv] */
  const double*  escrd;      /* [esmax] self-energy mesh (may be NULL if selfcal == 0) */
} ermod_mesh;

/* &hist namelist (engproc.F90:68-70). */
typedef struct ermod_hist {
  double ecdmin, ecfmns, ecdcen, eccore, ecdmax;
  double eclbin, ecfbin, ec0bin, finfac;
  int32_t pecore;
} ermod_hist;

/* Per-division accumulators (engmain.F90:327-347), fetched by engstore. */
typedef struct ermod_accum {
  double* edens;      /* [ermax] */
  double* ecorr;      /* [ermax*ermax] column-major, or NULL */
  double* eself;      /* [esmax] or NULL */
  float*  slnuv;      /* [numslv] soln only, or NULL */
  float*  minuv;      /* [numslv+1], index 0 = self energy */
  float*  maxuv;      /* [numslv+1] */
  double  avslf, engnorm, engsmpl, voffset;
  int32_t voffset_initialized;
} ermod_accum;

typedef struct ermod_ctx ermod_ctx;

/* Learned insertion proposal: network size (no reference counterpart). */
#define ERMOD_MLP_IN       64     /* 4x4x4 local solvent-density inputs */
#define ERMOD_MLP_HIDDEN   128    /* width of the three hidden layers */
#define ERMOD_MLP_NPARAMS  41473  /* W1[128][64] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] w4[128] b4 */

/* ABI version (ERMOD_ABI_VERSION). */
int32_t ermod_abi_version(void);

/*
 * enginit's energy-coordinate mesh (engproc.F90:171-226, 264-281) for
 * `numslv` species sharing one &hist set, without EcdInfo/EcdMesh files.
 * Outputs may be NULL to query sizes: *ermax, *esmax, *pemax, *pesoft.
 * uvcrd needs numslv*pemax entries, escrd pesoft entries.
 */
int32_t ermod_enginit_mesh(const ermod_hist* hist, int32_t numslv,
                           double* uvcrd, int32_t* uvmax, int32_t* uvsoft,
                           double* escrd, int32_t* ermax, int32_t* esmax);

/*
 * Create a context on CUDA device `device`.  Copies everything it needs;
 * the caller's arrays may be freed afterwards.  Replaces the one-time
 * setup done by enginit (engproc.F90:36-319), recpcal_init
 * (recpcal.F90:40-95) and instslt('init') (insertion.F90:48-62).
 */
int32_t ermod_create(ermod_ctx** out, int32_t device, const ermod_params* params,
                     const ermod_topology* topo, const ermod_mesh* mesh);

/*
 * RefInfo reference structure (load_refstructure, erdst/insertion.F90:676-770)
 * for insposition 5 (RMSD) and 6 (Gaussian): each frame, the reference host
 * is fitted onto the frame's host atoms and the reference solute carried
 * along (reffit, :646-673; fit_a_rotate_b, erdst/bestfit.F90:309-336); that
 * best-fit solute is the insertion origin and the RMSD reference
 * (check_solute_configuration :617-643, check_mol_configuration
 * erdst/engproc.F90:1249-1269 for solutes in solution).
 *   refspec   bit (sp - 1) set for each solvent species sp (uvspec) of the host
 *   nhost     the atoms of the refspec molecules, in molecule order
 *   host_crd  [3*nhost] their reference coordinates, host_w [nhost] fit weights
 *   slt_crd   [3*s] the reference solute coordinates, slt_w [s] its weights
 * Copies the arrays.  Call after ermod_create, before the first frame.
 */
int32_t ermod_set_refstructure(ermod_ctx* ctx, int32_t refspec, int32_t nhost, const float* host_crd,
                               const float* host_w, const float* slt_crd, const float* slt_w);

/* engclear (engproc.F90:321-340): zero the per-division accumulators. */
int32_t ermod_engclear(ermod_ctx* ctx);

/*
 * engconst (engproc.F90:353-517) for one frame.
 *   sitepos             [3*numatm_phys]: coordinates of the physical atoms
 *                       (solvent + soln solute) as read by getconf_parallel
 *                       (setconf.F90:849-986); the test particle is NOT included.
 *   cell                [9] column-major cell vectors (engmain.F90:323).
 *   stat_weight_system  frame weight (setconf.F90:974).
 *   ins_conf            refs only: NULL = rigid bfcoord for every insertion;
 *                       else [3*s*maxins] per-insertion solute coordinates
 *                       (what getsolute reads from SltConf, insertion.F90:393-543),
 *                       to which insposition / insorient are then applied.
 *   ins_weight          refs only: NULL = 1.0, else [maxins] per-insertion
 *                       structure weight (insertion.F90:541-542).
 *   flceng              soln only: [numslv*numslt] per-solute energy sums
 *                       (engproc.F90:918,932), or NULL.
 */
int32_t ermod_engconst(ermod_ctx* ctx, int32_t stnum, const float* sitepos,
                       const float* cell, float stat_weight_system,
                       const float* ins_conf, const float* ins_weight,
                       float* flceng);

/* Same as ermod_engconst with the inputs already in device memory. */
int32_t ermod_engconst_dev(ermod_ctx* ctx, int32_t stnum, const float* sitepos_dev,
                           const float* cell, float stat_weight_system,
                           const float* ins_conf_dev, const float* ins_weight_dev);

/*
 * Raw accumulators of the current division (engstore's inputs,
 * engproc.F90:578-604, before normalisation).  NULL members are skipped.
 */
int32_t ermod_fetch_accum(ermod_ctx* ctx, ermod_accum* out);

/*
 * engstore normalisation (engproc.F90:609-628): edens, ecorr and eself
 * divided by engnorm, avslf / engnorm, and the two avediv entries
 * avediv(division,1) = engnorm/engsmpl,
 * avediv(division,2) = voffset -/+ temp*log(avslf)  (soln / refs).
 * Writes the normalised arrays into `out` (same members as ermod_fetch_accum;
 * in soln mode `slnuv` receives aveuv = slnuv / engnorm, engproc.F90:622)
 * and avediv[2].  Does not clear the accumulators (call ermod_engclear).
 */
int32_t ermod_engstore(ermod_ctx* ctx, ermod_accum* out, double* avediv);

/*
 * Per-molecule energies of the last engconst call, the reference's
 * uvengy(slvmax, maxdst) and uvengy0(maxdst) (engproc.F90:369-370,
 * 442-457) in FP64.  uvengy is column-major: molecule index fastest,
 * molecules in tagpt order (physical molecules in input order).
 * Either pointer may be NULL.
 */
int32_t ermod_get_uvengy(ermod_ctx* ctx, double* uvengy, double* uvengy0);

/*
 * Solute coordinates of every insertion of the last engconst call
 * ([3*s*maxins], the reference's sitepos(:, numatm+1 ...) copies written
 * by instslt, insertion.F90:100-375) and the per-insertion importance
 * weights ([maxins], 1.0 for uniform insertion).  Either may be NULL.
 */
int32_t ermod_get_insertions(ermod_ctx* ctx, float* ins_sitepos, double* ins_weight);

/* Sizes: slvmax, maxdst, number of solute sites s, numatm_phys. */
int32_t ermod_get_sizes(ermod_ctx* ctx, int32_t* slvmax, int32_t* maxdst,
                        int32_t* nsite_solute, int32_t* numatm_phys);

/* The reference's 7-char error code of the last failing call ("" if none). */
const char* ermod_last_error(const ermod_ctx* ctx);

/* Device time (ms) of the stages of the last engconst, measured with CUDA
 * events on the engine's stream (no reference counterpart; profiling):
 * [0] total, [1] prepare + cell list, [2] insertion, [3] real space,
 * [4] PME spread, [5] FFT R2C, [6] influence multiply, [7] FFT C2R,
 * [8] PME gather, [9] binning, [10] weights + edens, [11] ecorr,
 * [12] number of PME target chunks, [13] potential-grid transpose,
 * [14] fused solve: stencil transforms, spectrum planes and 2-D FFTs,
 * [15] fused solve: k1 transforms into the potential grids, [16] fused
 * solve: per-site stencil transforms of a batch.  n <= 17. */
int32_t ermod_get_timings(const ermod_ctx* ctx, float* ms, int32_t n);

/* The PME solve the context runs (1..3 as ermod_params.spectrum_path, 0 when
 * there is no reciprocal-space term) and the ecorr kernel (0 tensor-core
 * GEMM, 1 FP64 kernel, -1 no ecorr); resolves the automatic choices (no
 * reference counterpart). */
int32_t ermod_get_paths(const ermod_ctx* ctx, int32_t* spectrum_path, int32_t* ecorr_path);

/* Kernel launches of this library since the context was created, cuFFT's
 * own kernels excluded (no reference counterpart; profiling). */
int64_t ermod_get_launch_count(const ermod_ctx* ctx);

void ermod_destroy(ermod_ctx* ctx);

/*
 * Batches of solutes sharing one solvent frame (no reference counterpart).
 * `members` are contexts created by ermod_create on one device for the same
 * solvent (same numatm_phys), each with its own solute, insertion count and
 * options.  ermod_batch_engconst runs the frame of every member as ONE
 * CUDA-graph launch with a branch per member; each member's results are
 * bit-identical to calling ermod_engconst on that member alone with the
 * same inputs, and are read with the member functions (ermod_fetch_accum,
 * ermod_engstore, ermod_get_uvengy, ...).  Refs-mode members use their rigid
 * solute (no per-insertion conformations).  The batch does not own the
 * members; destroy it before them.
 */
/*
 * Learned insertion proposal (refs mode, insposition random; no reference
 * counterpart).  The cell is cut into G^3 voxels (G = voxels_per_side) and,
 * for the network's inputs, into F^3 feature cells (F = feature_cells,
 * 0: 2G): a voxel's inputs are the 4x4x4 feature cells nearest its centre;
 * with ermod_params.proposal == ERMOD_PROPOSAL_LEARNED an insertion's
 * voxel is drawn from q_v = mix_uniform / G^3 + (1 - mix_uniform) *
 * softmax(s)_v, s_v the network's logit from the voxel's 4x4x4 local
 * density of solvent first sites, the point inside the voxel uniformly, and
 * the insertion's weight is multiplied by p/q = 1 / (G^3 q_v).  `params`
 * (ERMOD_MLP_NPARAMS FP32, layout above; weight matrices are used rounded
 * to BF16) may be NULL to only record voxels and features with uniform
 * insertion (training data).  mix_uniform in (0, 1].
 */
int32_t ermod_proposal_config(ermod_ctx* ctx, int32_t voxels_per_side, int32_t feature_cells, float mix_uniform,
                              const float* params);
/* Per insertion of the last frame: its voxel's 64 network inputs
 * ([maxdst*64]), its total solute-solvent energy ([maxdst]) and its voxel
 * index ([maxdst]); any pointer may be NULL. */
int32_t ermod_get_insertion_samples(ermod_ctx* ctx, float* features, double* etot, int32_t* voxel);

/*
 * The proposal network's trainer: hand-written forward, backward and Adam
 * kernels on one device (no reference counterpart).  The forward pass runs the
 * three hidden layers on the tensor cores (TF32 inputs, rounded to nearest with
 * ties away from zero; BF16 weights; FP32 accumulation), the backward pass and
 * Adam on the CUDA cores.  Loss: mean binary cross-entropy of the logit against
 * labels y in [0, 1].  Batches are host arrays x[n*64], y[n], n <= max_batch.
 */
typedef struct ermod_mlp ermod_mlp;
int32_t ermod_mlp_create(ermod_mlp** out, int32_t device, int32_t max_batch, const float* init_params);
int32_t ermod_mlp_nparams(void);
int32_t ermod_mlp_forward(ermod_mlp* m, const float* x, int32_t n, float* logits);
/* The hidden activations act[3][n][128] (after bias and ReLU, FP32) of the last
 * forward or gradient pass, which ran over n samples. */
int32_t ermod_mlp_activations(ermod_mlp* m, int32_t n, float* act);
int32_t ermod_mlp_gradients(ermod_mlp* m, const float* x, const float* y, int32_t n, float* grad, double* loss);
int32_t ermod_mlp_train_step(ermod_mlp* m, const float* x, const float* y, int32_t n, float lr, double* loss);
int32_t ermod_mlp_get_params(ermod_mlp* m, float* params);
void ermod_mlp_destroy(ermod_mlp* m);

typedef struct ermod_batch ermod_batch;
int32_t ermod_batch_create(ermod_batch** out, int32_t n, ermod_ctx* const* members);
int32_t ermod_batch_engconst(ermod_batch* b, int32_t stnum, const float* sitepos, const float* cell,
                             float stat_weight_system);
int32_t ermod_batch_engconst_dev(ermod_batch* b, int32_t stnum, const float* sitepos_dev, const float* cell,
                                 float stat_weight_system);
/* Device time (ms) of the last batch frame, CUDA events around the graph launch. */
float ermod_batch_last_ms(const ermod_batch* b);
/* "member <i>: <code>" for the first member that failed in the last call, "" if none. */
const char* ermod_batch_last_error(const ermod_batch* b);
void ermod_batch_destroy(ermod_batch* b);

/*
 * Energy histogram without device allocation.  No counterpart in the
 * reference: it serves hosts that may not allocate GPU memory themselves,
 * e.g. a Fortran erdst whose device memory belongs to its OpenACC runtime,
 * or an MPI rank held to a fixed GPU memory budget by its scheduler.
 *
 * Bins the per-molecule energies uvengy (host, [ntarget*nmol], molecule
 * fastest, as returned by ermod_get_uvengy) with getiduv's rule and returns
 * edens(i) = sum over targets of weight(target) * count(target, i) (host,
 * [ermax] with ermax = sum(uvmax)).  uvspec [nmol] gives each molecule's
 * solvent species (a 0 is an error, eng_cns, as in the engine), uvcrd /
 * uvmax / uvsoft the mesh (uvsoft may be NULL; it is used only when
 * slttype == ERMOD_SLT_SOLN).  Status codes as ermod_engconst.
 *
 * Solutes in solution (slttype == ERMOD_SLT_SOLN): the engine skips the
 * solute's own molecule (its uvspec is 0).  Here every column of uvengy is
 * binned, so leave the solute's column out of uvengy and its entry out of
 * uvspec (nmol one less than the physical molecule count).
 *
 * All device memory it uses is one array of ERMOD_NOALLOC_SCRATCH_BYTES
 * compiled into the library, which every GPU that loads the library holds
 * until the process exits; requests that do not fit return
 * ERMOD_ERR_OVERFLOW.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress) and keeps it for later calls; make
 * that first call before any stream capture.  The kept address belongs to
 * the device's current context: after cudaDeviceReset it is stale, so do not
 * call this entry point again in that process.  Calls run on the legacy
 * default stream and share the one array: calls that overlap on the GPU
 * (other host threads, other streams) race and must be serialised by the
 * caller.
 */
#define ERMOD_NOALLOC_SCRATCH_BYTES (32u << 20)
int32_t ermod_histogram_noalloc(int32_t device, int32_t slttype, const double* uvengy, int32_t ntarget,
                                int32_t nmol, const int32_t* uvspec, const double* uvcrd,
                                const int32_t* uvmax, const int32_t* uvsoft, int32_t numslv,
                                const double* weight, double* edens);

#ifdef __cplusplus
}
#endif
#endif /* ERMOD_B200_H */
