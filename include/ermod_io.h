/*
 * ermod_io.h -- erdst's on-disk formats, host side, in the same library as
 * the engine (libermod_b200.so).  No GPU is used by anything declared here.
 *
 *   trajectory reading   replaces vmdfio.c:132-385 (the VMD molfile plugin
 *                        path that trajectory.F90 binds) for CHARMM / NAMD /
 *                        X-PLOR DCD files: HISTORY (getconf_parallel,
 *                        setconf.F90:849-986) and SltConf (getsolute,
 *                        insertion.F90:393-543).
 *   engstore's files     engproc.F90:630-722: aveuv.tt, weight_soln /
 *                        weight_refs, uvrange.tt, engsln / engref,
 *                        corsln / corref (Fortran unformatted), slfeng.
 *
 * Conventions are those of ermod_b200.h: plain C types, caller-owned host
 * arrays in the reference's column-major layout, 0 = success, < 0 = error
 * with a 7-character name from ermod_io_last_error().
 */
#ifndef ERMOD_IO_H
#define ERMOD_IO_H

#include <stdint.h>

#include "ermod_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ERMOD_ERR_IO        (-30)  /* file missing, unreadable or not writable */
#define ERMOD_ERR_FORMAT    (-31)  /* not a DCD file, or a record of the wrong size */
#define ERMOD_TRJ_EOF       1      /* read_trajectory's non-zero status at the end */

typedef struct ermod_traj ermod_traj;

/*
 * open_trajectory (trajectory.F90:39-52 over vmdfio_open_traj_): opens a DCD
 * file in either byte order, with 32- or 64-bit record markers.  *natoms
 * receives the atom count of the file, *nframes the frame count of its header
 * (0 when the writer did not fill it in), *has_cell 1 when every frame carries
 * a unit-cell record.  Files with fixed atoms (NAMNF != 0) are refused
 * ("trj_fix"), as the plugin's reader of free atoms is not part of this path.
 */
int32_t ermod_traj_open(const char* path, ermod_traj** out, int32_t* natoms, int32_t* nframes,
                        int32_t* has_cell);

/*
 * read_trajectory (trajectory.F90:67-91 over vmdfio_read_traj_step_,
 * vmdfio.c:303-385): the next frame's coordinates crd[3*natoms] (x, y, z per
 * atom, Angstrom) and the cell cell[9] (column-major cell vectors, a along x,
 * b in the xy plane, as vmdfio.c builds them from A, B, C, alpha, beta, gamma;
 * all zero when the file has no cell).  natoms must equal the file's count.
 * Returns 0, ERMOD_TRJ_EOF past the last frame, ERMOD_ERR_ARG ("trj_nat") on
 * an atom-count mismatch (vmdfio.c:316-321), or ERMOD_ERR_FORMAT on a
 * truncated record.
 */
int32_t ermod_traj_read(ermod_traj* t, int32_t natoms, float* crd, float* cell);

/* Back to the first frame (OUTconfig's wrap-around of SltConf, setconf.F90:106-116). */
int32_t ermod_traj_rewind(ermod_traj* t);

/* close_trajectory (trajectory.F90:55-61). */
void ermod_traj_close(ermod_traj* t);

/*
 * What engstore writes for one division.  `division` runs 1..engdiv; the
 * files of the last division (division == engdiv) add aveuv.tt (soln),
 * weight_soln / weight_refs and uvrange.tt.  Mesh arrays are enginit's
 * (ermod_enginit_mesh); uvmax / uvsoft are per species, 1-based counts.
 */
typedef struct ermod_store_info {
  int32_t slttype, corrcal, selfcal, wgtslf;
  int32_t division, engdiv;
  int32_t numslv, ermax, esmax;
  const double* uvcrd;     /* [ermax] */
  const int32_t* uvmax;    /* [numslv] */
  const int32_t* uvsoft;   /* [numslv] */
  const double* escrd;     /* [esmax] */
} ermod_store_info;

/*
 * engstore's writes (engproc.F90:630-722) into directory `dir`, from the
 * normalised accumulators of ermod_engstore:
 *   norm->edens [ermax], norm->ecorr [ermax*ermax] (corrcal), norm->eself
 *   [esmax] (selfcal), norm->minuv / maxuv [numslv+1];
 *   avediv [engdiv*2] column-major avediv(division, 1:2) of every division so far;
 *   aveuv [engdiv*numslv] column-major aveuv(division, species) (soln, else NULL).
 * Text files use the reference's edit descriptors as gfortran prints them
 * (g15.7, g25.15, e20.8, f15.5, i5, ...); corsln / corref is one gfortran
 * unformatted sequential record of ermax*ermax FP64 values with 4-byte
 * length markers in the machine's byte order.
 */
int32_t ermod_write_engstore(const char* dir, const ermod_store_info* info, const ermod_accum* norm,
                             const double* avediv, const float* aveuv);

/*
 * One value through a Fortran output edit descriptor as engstore's files use
 * them: kind 0 Gw.d, 1 Ew.d, 2 Fw.d, 3 Iw (x truncated to an integer).  Writes
 * the w-character field and a terminating NUL into out[cap].
 */
int32_t ermod_io_format(int32_t kind, double x, int32_t w, int32_t d, char* out, int32_t cap);

/*
 * rmsd_bestfit (bestfit.F90:339-346): the weighted RMSD of crd[3*n] from
 * ref[3*n] after the best rigid superposition of crd onto ref (weights w[n]),
 * as getsolute's insstructure filter uses it (insertion.F90:491-499).
 * Returns -1 when the weights sum to zero ('bst_zrw').
 */
double ermod_rmsd_bestfit(int32_t n, const float* ref, const float* crd, const float* w);

/* Name of the last error of the I/O entry points on this thread ("trj_opn", ...). */
const char* ermod_io_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ERMOD_IO_H */
