/* C++ host side of the drop-in path (part of libgegs_b200.so): a plan in the
 * reference's input formats read into the structs the transport calls take,
 * and the dose file written the way the reference writes it. A C or C++
 * caller drives a whole plan without Python:
 *
 *   gegs_plan_load(ini, physics file)  ->  gegs_create / gegs_set_physics /
 *   gegs_set_scene / gegs_run  ->  gegs_get_tally  ->  gegs_plan_dose  ->
 *   gegs_plan_write_dose
 *
 * Mapping to the reference (RicciWoo/GEGS):
 *   gegs_plan_load replaces main()'s INI parsing (CUDA_EGS.cu:907-1694,
 *     GetPrivateProfileString) and init() (init.cu:1682-1710): the egsphant
 *     phantom (init.cu:1164-1275), the regions' media and densities
 *     (init.cu:909-1052), the CM DYNVMLC and CM JAWS/SECJAWS blocks of the
 *     egsinp file (init.cu:345-689), the mlcinfo field list and the mlcinp leaf
 *     positions (read_mlcinp, init.cu:1377-1500), the per-field jaw and
 *     leaf-end polygons (setup_secjaws, init_leaf_pos, init.cu:1504-1662), the
 *     phase space (read_egsphsp.cpp:44-232), histories per field and phase-space
 *     recycling (runSimulation, CUDA_EGS.cu:377-391), the dose unit and the
 *     calibration (CUDA_EGS.h:536, CUDA_EGS.cu:1478);
 *   gegs_plan_dose / gegs_plan_write_dose replace write_dose (output.c:873-918).
 *
 * The physics tables come from a physics file, the reference's PEGS4/EGSnrc
 * data being absent: `python -m gegs_b200 -i plan.ini --write-physics FILE`
 * writes one for the plan's media. Its layout:
 *   bytes 0-7      "GEGSPHY1"
 *   bytes 8-11     uint32 sizeof(gegs_physics)
 *   bytes 12-15    uint32 nmed
 *   16 + 32*k      the name of medium k, NUL-padded to 32 bytes (k < nmed)
 *   16 + 32*nmed   the gegs_physics block (little-endian, as in memory)
 * The media must be the plan's, in the plan's order: the phantom's media,
 * then the default medium and the jaws' and MLC's media where not already
 * listed (init.cu:1322-1352).
 *
 * Not handled here (the Python CLI does them after the dose): [Interpolation]
 * and the [Dose output] point and relative doses. Block and Wedge modules and
 * CTcreate from DICOM are refused with an error, as by the CLI.
 */
#ifndef GEGS_PLAN_H
#define GEGS_PLAN_H

#include <stddef.h>
#include <stdint.h>
#include "gegs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gegs_plan gegs_plan;

/* Read the plan `ini_path` and the physics file `physics_path`. Relative data
 * paths are taken from the INI file's directory; Windows separators are
 * accepted. max_histories_per_field > 0 caps each field's histories (0: none).
 * On error returns GEGS_ERR_ARG with a message in msg (may be NULL). */
gegs_status gegs_plan_load(const char *ini_path, const char *physics_path, uint64_t max_histories_per_field,
                           gegs_plan **out, char *msg, size_t msg_len);
void gegs_plan_free(gegs_plan *p);

/* Owned by the plan; valid until gegs_plan_free. */
const gegs_physics *gegs_plan_physics(const gegs_plan *p);
const gegs_scene *gegs_plan_scene(const gegs_plan *p);
uint64_t gegs_plan_histories(const gegs_plan *p);     /* all fields: run [0, histories) */
uint64_t gegs_plan_nvox(const gegs_plan *p);
double gegs_plan_dose_unit(const gegs_plan *p);       /* cGy per MeV/g, calibration included (a float value) */
int32_t gegs_plan_nfields(const gegs_plan *p);
double gegs_plan_output_factor(const gegs_plan *p, int32_t field);   /* 1 unless [Output factor] is on;
                                                                        0 for a field size outside its table */

/* The voxel masses in g, in float as the reference computes them: |(dx dy) dz| * density, 0 taken
 * as 1 (init.cu:1256-1271); nvox floats. */
gegs_status gegs_plan_voxel_mass(const gegs_plan *p, float *mass, uint64_t nvox);

/* Dose per voxel from the int64 tally (MeV * 2^30), as the reference's write_dose computes it
 * from the energy E (output.c:887-891): (float)E / mass * dose_unit, in float. */
gegs_status gegs_plan_dose(const gegs_plan *p, const int64_t *tally, float *dose, uint64_t nvox);

/* Write <output directory>/<output prefix>_DoseResults_NNNxNNNxNNN.bin (raw
 * float32, x fastest), creating the directory; the file name goes to path. */
gegs_status gegs_plan_write_dose(const gegs_plan *p, const float *dose, uint64_t nvox, char *path, size_t path_len);

#ifdef __cplusplus
}
#endif
#endif /* GEGS_PLAN_H */
