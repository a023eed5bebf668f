/*
 * ermod_slvfe.h -- slvfe's free-energy functional (chmpot, slvfe.F90:744-803 with
 * distnorm :1467-1542, getslncv :875-1001 and getinscv :1003-1232) for one data set on
 * the GPU in FP64, with slvfe's default options (sfemain.F90:22-64): functional py-hnc,
 * invmtrx 'reg' (Cholesky, with getinscv's eigen-decomposition fallback), zerosft 'eczr',
 * wgtfnform 'harm', extsln 'lin', normalize 'yes'.  Same library and conventions as
 * ermod_b200.h.
 */
#ifndef ERMOD_SLVFE_H
#define ERMOD_SLVFE_H

#include <stdint.h>

#include "ermod_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ERMOD_ERR_SLVFE     (-40)  /* the functional cannot be evaluated on these distributions */

/*
 * rho_sln [n]   the solution distribution as engsln's ratio column holds it
 * rho_ref [n]   the reference-solvent distribution (engref's ratio column)
 * chi_ref [n*n] the reference-solvent correlation matrix (corref), column-major
 * crd [n]       bin coordinates (engsln's bin_middle), spec [n] 1-based species, each
 *               species' bins contiguous and in order
 * group         bins merged per species first (chmpot's grouping with inft 0,
 *               slvfe.F90:609-698; the reference reports group 3 in its range / merge
 *               modes, sfemain.F90:55); 1 = the mesh as read
 * inft          percentage (0..100) of each species' core bins (rduvcore, counted from
 *               crd as datread does) that join its last merged bin (slvfe.F90:613-615)
 * kT            kcal/mol (temp * 8.314510e-3 / 4.184, slvfe.F90:272)
 * aveuv [nsp]   average solute-solvent energy per species in solution
 * slfeng        solute self energy (slfslt 'yes'), else 0
 * Writes chmpt[nsp] (per-species free energies, aveuv included) and *total
 * (their sum + slfeng).  ERMOD_ERR_SLVFE with ermod_slvfe_last_error():
 *   "slv_nrm" chi0 normalisation did not converge in 100 sweeps;
 *   "slv_ext" a solution-side bin has no sampled neighbour to extrapolate from;
 *   "slv_chl" the solve failed: the eigen-decomposition fallback failed too, or
 *             (ermod_slvfe_delta_mu_ex with evd = 0) the regularised Cholesky solve
 *             failed or was rejected;
 *   "slv_zer" a species' mesh has no bin pair around zero energy.
 * ERMOD_ERR_ARG "slv_grp" when a species has fewer bins than `group`.
 */
int32_t ermod_slvfe_delta_mu(int32_t device, int32_t n, int32_t nsp, int32_t group, int32_t inft,
                             const double* rho_sln,
                             const double* rho_ref, const double* chi_ref, const double* crd,
                             const int32_t* spec, double kT, const double* aveuv, double slfeng,
                             double* chmpt, double* total);

/*
 * The same with slvfe's functional and solver options (no defaults changed by the
 * plain entry point above, which is opts = {ERMOD_SLVFE_PYHNC, 1, 0.0}):
 *   functional  chmpot's integrand (slvfe.F90:759-774): py-hnc (sfemain.F90:40), hnc,
 *               thnc with threshold et (thnc :1417-1436; sfemain.F90:177 picks thnc
 *               when et != 0), or none
 *   evd         1: when the regularised Cholesky solve fails, or posv_wrap's check
 *               rejects its solution (residual above 1e-6 or an element above 1e6,
 *               slvfe.F90:478, 520-531), solve by the eigen-decomposition of the
 *               unregularised matrix as getinscv does (:1124-1170; cuSOLVER Dsyevd, the
 *               reference's syevr_wrap :536-584); 0: report "slv_chl" instead
 *   *used_evd   (may be NULL) set to 1 when the eigen-decomposition gave the solution
 */
#define ERMOD_SLVFE_PYHNC 0
#define ERMOD_SLVFE_HNC   1
#define ERMOD_SLVFE_THNC  2
#define ERMOD_SLVFE_NONE  3
typedef struct ermod_slvfe_opts {
  int32_t functional;
  int32_t evd;
  double  et;
} ermod_slvfe_opts;

int32_t ermod_slvfe_delta_mu_ex(int32_t device, int32_t n, int32_t nsp, int32_t group, int32_t inft,
                                const double* rho_sln, const double* rho_ref, const double* chi_ref,
                                const double* crd, const int32_t* spec, double kT, const double* aveuv,
                                double slfeng, const ermod_slvfe_opts* opts, double* chmpt, double* total,
                                int32_t* used_evd);

/* Name of the last error of ermod_slvfe_delta_mu on this thread. */
const char* ermod_slvfe_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ERMOD_SLVFE_H */
