/* Dose post-processing and phantom preparation on the GPU (libgegs_b200.so).
 *
 * Each call takes host buffers, allocates device memory for its own use,
 * and returns 0 on success, 1 for an invalid argument, 2 for a CUDA error
 * and 5 when device memory runs out.
 */
#ifndef GEGS_POST_H
#define GEGS_POST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Dose at the points of a regular output grid (origin x0,y0,z0; spacing
 * sx,sy,sz; mx*my*mz points, x fastest) by linear interpolation in z, then y,
 * then x between voxel centres; points at or beyond the first or last centre
 * get 0. Replaces interp_dose (output.c:221-316), whose result file is the
 * dims (3 x int32) followed by the float32 grid. */
int gegs_interp_dose(int device, const float *dose, int nx, int ny, int nz, const float *x_bounds,
                     const float *y_bounds, const float *z_bounds, float x0, float y0, float z0, float sx,
                     float sy, float sz, int mx, int my, int mz, float *out);

/* 3-D global gamma index (no counterpart in the reference, whose comparison
 * with measured data is a 1-D/2-D check in output_RelDos_II): for every
 * reference voxel with dose >= cutoff_abs, gamma = min over evaluated voxels
 * within search_dta * dta of sqrt(r^2 / dta^2 + (E - R)^2 / dd_abs^2), on the
 * voxel grid (spacing dx, dy, dz; no sub-voxel interpolation). gamma[] gets -1
 * below the cutoff. n_evaluated / n_passed count the voxels compared and those
 * with gamma <= 1. */
int gegs_gamma3d(int device, const float *ref, const float *eval, int nx, int ny, int nz, float dx, float dy,
                 float dz, float dta, float dd_abs, float cutoff_abs, float search_dta, float *gamma,
                 uint64_t *n_evaluated, uint64_t *n_passed);

/* One segment of a CT ramp: HU in (previous upper, hu_upper] maps to medium
 * with density linear from density_lower to density_upper. */
typedef struct gegs_ct_ramp_segment {
    double hu_upper;
    double density_lower, density_upper;
    int32_t medium;
    int32_t pad_;
} gegs_ct_ramp_segment;

/* HU -> medium index and density (g/cm^3) per voxel (CTToMedium's ramp,
 * ctcreate.c:913-970 and 1057-1104): HU below hu_lower -> medium 0xFFFF
 * (vacuum), density 0; above the last segment -> its medium at its upper
 * density. */
int gegs_ct_ramp(int device, const int16_t *hu, uint64_t n, const gegs_ct_ramp_segment *segments, int nseg,
                 double hu_lower, uint16_t *medium, float *density);

#ifdef __cplusplus
}
#endif
#endif /* GEGS_POST_H */
