/* Entry points of the reference-pinning harness (test infrastructure). */
#ifndef GEGS_REF_API_H
#define GEGS_REF_API_H
#include <stdint.h>
#include "../../include/gegs_physics.h"
#include "../../include/gegs_scene.h"
#include "../gegs_oracle.h"        /* gegs_probe_particle */

#ifdef __cplusplus
extern "C" {
#endif
int ref_load(const gegs_physics *P, const gegs_scene *S);
int ref_select_field(int f);
int ref_probe_geom(uint32_t n, const gegs_probe_particle *in, const float *t_in, uint32_t *far_region,
                   float *far_t, gegs_probe_particle *far_out, float *near_t);
int ref_probe_uphi(int which, float a, float b, gegs_probe_particle *p, float *cs, float u);
int ref_probe_stage(int stage, uint32_t n, const gegs_probe_particle *in, const float *u, const uint32_t *un,
                    uint32_t ucap, gegs_probe_particle *out, uint32_t ocap, uint32_t *on, uint32_t *dreg, float *de,
                    uint32_t dcap, uint32_t *dn, uint32_t *used);
/* host set-up: the reference's readers on plan files (init.cu); outfac_file NULL = off */
int ref_setup_run(const char *egsphant, const char *mlc_egsinp, const char *jaws_egsinp, const char *mlcinfo,
                  const char *data_directory, const char *outfac_file, float sid, const char *default_medium,
                  char *msg, size_t msg_len);
long ref_setup_get(const char *name, int field, void *dst, size_t bytes);
/* a whole transport of histories [h0, h1) of the loaded scene by the reference's kernels */
long ref_transport(uint64_t h0, uint64_t h1, uint64_t seed, double *tally, uint64_t nvox);
#ifdef __cplusplus
}
#endif
#endif
