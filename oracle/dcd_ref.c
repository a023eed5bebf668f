/*
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE: a C shim that drives the reference's
 * own DCD reader -- the VMD molfile plugin the reference vendors as source
 * (vmdplugins/dcdplugin.c) and loads through vmdfio.c -- so that the tests can
 * compare the library's DCD reader with it frame by frame.  Built by
 * `make ref` into oracle/_ref/ only where the reference sources are present.
 */
#include <string.h>

#include "molfile_plugin.h"

extern int molfile_dcdplugin_init(void);
extern int molfile_dcdplugin_register(void *v, vmdplugin_register_cb cb);

static molfile_plugin_t *plugin_ = NULL;

static int take(void *v, vmdplugin_t *p) {
  (void)v;
  plugin_ = (molfile_plugin_t *)p;
  return 0;
}

int ref_dcd_init(void) {
  if (plugin_) return 0;
  molfile_dcdplugin_init();
  molfile_dcdplugin_register(NULL, take);
  return plugin_ ? 0 : -1;
}

void *ref_dcd_open(const char *path, int *natoms) {
  if (ref_dcd_init() != 0) return NULL;
  *natoms = MOLFILE_NUMATOMS_UNKNOWN;
  return plugin_->open_file_read(path, "dcd", natoms);
}

/* one frame: crd[3*natoms] and the timestep's A, B, C, alpha, beta, gamma as the plugin fills
   them (vmdfio.c:303-385 builds the cell from these); 0, or 1 past the last frame */
int ref_dcd_read(void *h, int natoms, float *crd, float *abc_angles) {
  molfile_timestep_t ts;
  memset(&ts, 0, sizeof(ts));
  ts.coords = crd;
  if (plugin_->read_next_timestep(h, natoms, &ts) != MOLFILE_SUCCESS) return 1;
  abc_angles[0] = ts.A; abc_angles[1] = ts.B; abc_angles[2] = ts.C;
  abc_angles[3] = ts.alpha; abc_angles[4] = ts.beta; abc_angles[5] = ts.gamma;
  return 0;
}

void ref_dcd_close(void *h) { plugin_->close_file_read(h); }
