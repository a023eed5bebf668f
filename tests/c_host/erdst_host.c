/*
 * erdst_host.c -- a plain C host of the engine library, with no Python: it
 * replays trjmain's per-division sequence (erdst/enganal.F90:54-106) over the
 * C-ABI of include/ermod_b200.h:
 *
 *   ermod_enginit_mesh  (enginit's mesh, engproc.F90:171-281)
 *   ermod_create        (enginit / recpcal_init / instslt('init'))
 *   ermod_engclear      (engclear, engproc.F90:321-340)
 *   ermod_engconst x N  (engconst(stnum) per frame, engproc.F90:353-517)
 *   ermod_engstore      (engstore's normalisation, engproc.F90:609-628)
 *
 * Input (argv[1]): a flat little-endian record written by the test:
 *   int32  nummol, numatm, ljtype_max, nsite, numatm_phys, nframes, numslv, device
 *   int32  numsite[nummol], sluvid[nummol], uvspec[nummol]
 *   float  charge[numatm]; int32 ljtype[numatm]; float sitemass[numatm]
 *   float  ljene[ljtype_max^2], ljlensq[ljtype_max^2], bfcoord[3 nsite]
 *   bytes  ermod_params, ermod_hist (as the header lays them out)
 *   per frame: float sitepos[3 numatm_phys], float cell[9]
 * Output (argv[2]): int32 status of each call, ermax, then double
 * edens[ermax] (normalised), avediv[2], engnorm, engsmpl, voffset.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ermod_b200.h"

static FILE* in;

static void* rd(size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (!p || (bytes && fread(p, 1, bytes, in) != bytes)) {
    fprintf(stderr, "short input\n");
    exit(2);
  }
  return p;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s input output\n", argv[0]);
    return 2;
  }
  in = fopen(argv[1], "rb");
  if (!in) return 2;
  int32_t* hdr = (int32_t*)rd(8 * sizeof(int32_t));
  const int nummol = hdr[0], numatm = hdr[1], ljmax = hdr[2], nsite = hdr[3], natp = hdr[4];
  const int nframes = hdr[5], numslv = hdr[6], device = hdr[7];
  ermod_topology topo;
  topo.nummol = nummol;
  topo.numsite = (const int32_t*)rd(sizeof(int32_t) * nummol);
  topo.sluvid = (const int32_t*)rd(sizeof(int32_t) * nummol);
  topo.uvspec = (const int32_t*)rd(sizeof(int32_t) * nummol);
  topo.charge = (const float*)rd(sizeof(float) * numatm);
  topo.ljtype = (const int32_t*)rd(sizeof(int32_t) * numatm);
  topo.sitemass = (const float*)rd(sizeof(float) * numatm);
  topo.ljtype_max = ljmax;
  topo.ljene_mat = (const float*)rd(sizeof(float) * ljmax * ljmax);
  topo.ljlensq_mat = (const float*)rd(sizeof(float) * ljmax * ljmax);
  topo.bfcoord = (const float*)rd(sizeof(float) * 3 * nsite);
  ermod_params* prm = (ermod_params*)rd(sizeof(ermod_params));
  ermod_hist* hist = (ermod_hist*)rd(sizeof(ermod_hist));

  int32_t st[8] = {0};
  int32_t ermax = 0, esmax = 0;
  st[0] = ermod_enginit_mesh(hist, numslv, NULL, NULL, NULL, NULL, &ermax, &esmax);
  double* uvcrd = (double*)calloc(ermax, sizeof(double));
  double* escrd = (double*)calloc(esmax ? esmax : 1, sizeof(double));
  int32_t* uvmax = (int32_t*)calloc(numslv, sizeof(int32_t));
  int32_t* uvsoft = (int32_t*)calloc(numslv, sizeof(int32_t));
  if (st[0] == 0) st[0] = ermod_enginit_mesh(hist, numslv, uvcrd, uvmax, uvsoft, escrd, &ermax, &esmax);
  ermod_mesh mesh = {numslv, ermax, esmax, uvcrd, uvmax, uvsoft, escrd};

  ermod_ctx* ctx = NULL;
  st[1] = ermod_create(&ctx, device, prm, &topo, &mesh);
  if (st[1] == 0) st[2] = ermod_engclear(ctx);
  float* pos = (float*)malloc(sizeof(float) * 3 * natp);
  float cell[9];
  for (int f = 0; f < nframes; ++f) {
    if (fread(pos, sizeof(float), 3 * natp, in) != (size_t)(3 * natp) || fread(cell, sizeof(float), 9, in) != 9) {
      fprintf(stderr, "short frame\n");
      return 2;
    }
    /* engconst(stnum): stnum counts frames from 1 (enganal.F90:88) */
    const int32_t rc = st[1] == 0 ? ermod_engconst(ctx, f + 1, pos, cell, 1.0f, NULL, NULL, NULL) : -1;
    if (rc < 0 && st[3] == 0) st[3] = rc;
    if (rc > 0 && st[3] == 0) st[3] = rc;   /* mbin: the reference warns and carries on */
  }
  fclose(in);

  double* edens = (double*)calloc(ermax, sizeof(double));
  double* ecorr = prm->corrcal ? (double*)calloc((size_t)ermax * ermax, sizeof(double)) : NULL;
  float* minuv = (float*)calloc(numslv + 1, sizeof(float));
  float* maxuv = (float*)calloc(numslv + 1, sizeof(float));
  double avediv[2] = {0, 0};
  ermod_accum acc;
  memset(&acc, 0, sizeof(acc));
  acc.edens = edens;
  acc.ecorr = ecorr;
  acc.minuv = minuv;
  acc.maxuv = maxuv;
  if (st[1] == 0) st[4] = ermod_engstore(ctx, &acc, avediv);
  if (st[1] != 0 || st[3] < 0 || st[4] != 0)
    fprintf(stderr, "failed: %s\n", ctx ? ermod_last_error(ctx) : "create");

  FILE* out = fopen(argv[2], "wb");
  if (!out) return 2;
  fwrite(st, sizeof(int32_t), 8, out);
  fwrite(&ermax, sizeof(int32_t), 1, out);
  fwrite(edens, sizeof(double), ermax, out);
  fwrite(avediv, sizeof(double), 2, out);
  fwrite(&acc.engnorm, sizeof(double), 1, out);
  fwrite(&acc.engsmpl, sizeof(double), 1, out);
  fwrite(&acc.voffset, sizeof(double), 1, out);
  fclose(out);
  if (ctx) ermod_destroy(ctx);
  return (st[0] | st[1] | st[2] | st[4]) != 0 || st[3] < 0;
}
