/* Input description of one transport job: phantom, beam-line geometry, fields
 * and phase-space source.  Plain C types only (no CUDA, no torch): the same
 * struct feeds the CUDA library (include/gegs.h) and the CPU oracle.
 *
 * Every field restates state the reference keeps in host statics and
 * __constant__/__device__ symbols:
 *   phantom bounds / voxel media / densities  init.cu:1164-1271, init.cu:909-1052
 *   change_xyz, source_to_isocenter, iso       CUDA_EGS.cu:1404-1452
 *   module order                               CUDA_EGS.cu:1277-1305
 *   MLC cross sections (crossXZ, boundaries)   init.cu:345-611 (read_egsinp)
 *   per-field jaw polygons                     init.cu:1504-1592 (setup_secjaws)
 *   per-field leaf-end polygons (endnode)      init.cu:1594-1662 (init_leaf_pos)
 *   gantry cos/sin                             CUDA_EGS.cu:426-434
 *   phase-space records (MODE0, 28 bytes)      read_egsphsp.h, CUDA_EGS.cu:40-158
 */
#ifndef GEGS_SCENE_H
#define GEGS_SCENE_H

#include <stdint.h>

#define GEGS_MAX_FIELDS 32
#define GEGS_N_LEAF_PAIRS 60
#define GEGS_VACUUM_MED 0xFFFFu

/* module numbers (CUDA_EGS.h:391-399) */
enum gegs_module {
    GEGS_M_FIRST = 0, GEGS_M_SECJAWY = 1, GEGS_M_SECJAWX = 2, GEGS_M_VARMLC = 3,
    GEGS_M_WEDGE = 4, GEGS_M_BLOCK = 5, GEGS_M_PHANTOM = 6
};

/* region flags (CUDA_EGS.h:567-576) */
enum gegs_region_flags {
    GEGS_F_RAYLEIGH = 0x0001u, GEGS_F_BOUND_COMPTON = 0x0002u,
    GEGS_F_ATOMIC_RELAXATION = 0x0010u, GEGS_F_PHOTO_ANGULAR = 0x0020u
};

/* One BEAMnrc MODE0 phase-space record (read_egsphsp.h: LATCH, E, X, Y, U, V, WT). */
typedef struct gegs_phsp_record {
    uint32_t latch;
    float e, x, y, u, v, wt;
} gegs_phsp_record;

/* Per-field beam-modifier state.  Polygons are (x, y) float pairs. */
typedef struct gegs_field {
    float cos_angle, sin_angle;            /* gantry rotation (float, as uploaded by the reference) */
    uint64_t hist_begin, hist_end;         /* global history range of this field */
    int32_t nrepeat;                       /* phase-space recycling: each record used nrepeat+1 times */
    int32_t pad_;
    float boundMinY[4][2], boundMinX[4][2];
    float boundMaxY[4][2], boundMaxX[4][2];
    float jawsGeomY[8][2], jawsGeomX[8][2];
    float endnode[GEGS_N_LEAF_PAIRS][34][2];
} gegs_field;

typedef struct gegs_scene {
    /* voxel phantom */
    int32_t nx, ny, nz;
    const float *x_bounds, *y_bounds, *z_bounds;   /* n+1 planes each */
    const uint16_t *voxel_med;                     /* medium index per voxel, GEGS_VACUUM_MED = vacuum */
    const float *voxel_rhof;                       /* density / standard medium density */
    int32_t other_med[5];                          /* media of regions 1..5: default, jaws, MLC, block, wedge */
    uint32_t region_flags;                         /* flags of every non-vacuum region */

    /* patient placement */
    int32_t change_xyz;
    float source_to_isocenter;
    float iso[3];
    float z_phsp;                                  /* z of the phase-space plane (beam frame) */
    int8_t module_order[8];                        /* next module after module m; [0] = first module */

    /* DYNVMLC (read_egsinp) */
    float mlc_rmax, mlc_zmin, mlc_zthick, mlc_x_start, mlc_x_end, mlc_x_mid_1, mlc_x_mid_2;
    float mlc_air_gap, mlc_wl_full, mlc_wl_target, mlc_wl_isocenter, mlc_wt;
    float crossXZ[960][2];
    float boundaryXZ[4][2], boundaryYZ[4][2];

    /* fields and source */
    int32_t nfields;
    const gegs_field *fields;
    const gegs_phsp_record *phsp;
    uint64_t nphsp;

    /* options */
    int32_t hownear_region_offset;   /* 5: reference voxel decode in hownear_phantom; 6: corrected */
    int32_t pad2_;
    uint64_t seed;                   /* Philox key */

    /* Beamlets (no counterpart in the reference): a grid of bl_nx x bl_ny
     * bixels of bl_dx x bl_dy cm starting at (bl_x0, bl_y0) in the isocentre
     * plane of the beam frame, the same for every field. A primary is tagged
     * with the bixel its straight line from the phase-space plane crosses;
     * beamlet index = field * bl_nx * bl_ny + iy * bl_nx + ix. Its weight is
     * multiplied by bl_weight[index] (NULL: weights 1). bl_nx = 0: no beamlets. */
    int32_t bl_nx, bl_ny;
    float bl_x0, bl_y0, bl_dx, bl_dy;
    const float *bl_weight;
} gegs_scene;

#endif /* GEGS_SCENE_H */
