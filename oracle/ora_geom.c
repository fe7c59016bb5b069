/* Oracle: geometry routines restated from geom.cu.  Test infrastructure only.
 *   isWhere            geom.cu:20-36
 *   howfar_phantom     geom.cu:54-307
 *   pointInPolygon ..  geom.cu:310-515   (MLC helpers)
 *   howfar_MLC         geom.cu:518-790
 *   howfar_SecJawsY/X  geom.cu:793-1035
 *   hownear_MLC ..     geom.cu:1152-1286
 *   hownear_SecJaws    geom.cu:1288-1374
 *   hownear_phantom    geom.cu:1422-1543
 * The reference's behaviour is kept, including the voxel decode of
 * hownear_phantom (region - 5, selectable through hownear_region_offset) and
 * the dis_yz step of howfar_SecJawsX inside the tungsten. */
#include "ora_internal.h"

typedef struct { float x, y; } pt2;

static inline pt2 P2(const float *a) { pt2 r = {a[0], a[1]}; return r; }

/* ---- phantom ------------------------------------------------------------ */
static int isWhere(float p, uint32_t nreg, const float *bounds)
{
    if ((p < bounds[0]) || (p > bounds[nreg])) return -1;
    if (nreg == 1) return 0;
    int ml = 0, mu = (int)nreg;
    while (mu - ml > 1) {
        int mav = (ml + mu) / 2;
        if (p <= bounds[mav]) mu = mav; else ml = mav;
    }
    return mu - 1;
}

typedef struct { float x, y, z, u, v, w; } ptr6;

static ptr6 to_patient(const ora_ctx *C, const ora_particle *p0)
{
    const gegs_scene *S = C->S;
    const gegs_field *F = &S->fields[p0->field];
    ptr6 p;
    if (S->change_xyz) {
        p.x = p0->y; p.y = p0->z - S->source_to_isocenter; p.z = p0->x;
        p.u = p0->v; p.v = p0->w; p.w = p0->u;
    } else {
        p.x = p0->x; p.y = p0->y; p.z = p0->z - S->source_to_isocenter;
        p.u = p0->u; p.v = p0->v; p.w = p0->w;
    }
    float tx = p.x * F->cos_angle - p.y * F->sin_angle;
    float ty = p.x * F->sin_angle + p.y * F->cos_angle;
    p.x = tx; p.y = ty;
    tx = p.u * F->cos_angle - p.v * F->sin_angle;
    ty = p.u * F->sin_angle + p.v * F->cos_angle;
    p.u = tx; p.v = ty;
    p.x = p.x + S->iso[0];
    p.y = p.y + S->iso[1];
    p.z = p.z + S->iso[2];
    return p;
}

uint32_t howfar_phantom(ora_ctx *C, const ora_particle *p0, float *t)
{
    const gegs_scene *S = C->S;
    const float *xb = S->x_bounds, *yb = S->y_bounds, *zb = S->z_bounds;
    uint32_t Nx = (uint32_t)S->nx, Ny = (uint32_t)S->ny, Nz = (uint32_t)S->nz;
    ptr6 p = to_patient(C, p0);
    uint32_t region = p0->region;
    if (region >= VAC_AND_OTH) {
        uint32_t ir = region - VAC_AND_OTH;
        int iz = (int)(ir / (Nx * Ny));
        ir -= (uint32_t)iz * Nx * Ny;
        int iy = (int)(ir / Nx);
        int ix = (int)(ir - (uint32_t)iy * Nx);
        uint32_t inew = region;
        if (p.u > 0.0f) {
            float d = (xb[ix + 1] - p.x) / p.u;
            if (d <= *t) { *t = d; if ((uint32_t)(++ix) < Nx) inew = region + 1; else inew = VACUUM_REG; }
        } else if (p.u < 0.0f) {
            float d = (xb[ix] - p.x) / p.u;
            if (d <= *t) { *t = d; if (--ix >= 0) inew = region - 1; else inew = VACUUM_REG; }
        }
        if (p.v > 0.0f) {
            float d = (yb[iy + 1] - p.y) / p.v;
            if (d <= *t) { *t = d; if ((uint32_t)(++iy) < Ny) inew = region + Nx; else inew = VACUUM_REG; }
        } else if (p.v < 0.0f) {
            float d = (yb[iy] - p.y) / p.v;
            if (d <= *t) { *t = d; if (--iy >= 0) inew = region - Nx; else inew = VACUUM_REG; }
        }
        if (p.w > 0.0f) {
            float d = (zb[iz + 1] - p.z) / p.w;
            if (d <= *t) { *t = d; if ((uint32_t)(++iz) < Nz) inew = region + Nx * Ny; else inew = VACUUM_REG; }
        } else if (p.w < 0.0f) {
            float d = (zb[iz] - p.z) / p.w;
            if (d <= *t) { *t = d; if (--iz >= 0) inew = region - Nx * Ny; else inew = VACUUM_REG; }
        }
        if (*t < 0) *t = EPSTEP;
        return inew;
    }
    int ix, iy, iz;
    float t1 = 0.0f;
    ix = -1;
    if ((p.x <= xb[0]) && (p.u > 0.0f)) { t1 = (xb[0] - p.x) / p.u; ix = 0; }
    else if ((p.x >= xb[Nx]) && (p.u < 0.0f)) { t1 = (xb[Nx] - p.x) / p.u; ix = (int)Nx - 1; }
    if ((ix >= 0) && (t1 <= *t)) {
        float y1 = p.y + p.v * t1;
        iy = isWhere(y1, Ny, yb);
        if (iy >= 0) {
            float z1 = p.z + p.w * t1;
            iz = isWhere(z1, Nz, zb);
            if (iz >= 0) { *t = t1; return (uint32_t)ix + (uint32_t)iy * Nx + (uint32_t)iz * Nx * Ny + VAC_AND_OTH; }
        }
    }
    iy = -1;
    if ((p.y <= yb[0]) && (p.v > 0.0f)) { t1 = (yb[0] - p.y) / p.v; iy = 0; }
    else if ((p.y >= yb[Ny]) && (p.v < 0.0f)) { t1 = (yb[Ny] - p.y) / p.v; iy = (int)Ny - 1; }
    if ((iy >= 0) && (t1 <= *t)) {
        float x1 = p.x + p.u * t1;
        ix = isWhere(x1, Nx, xb);
        if (ix >= 0) {
            float z1 = p.z + p.w * t1;
            iz = isWhere(z1, Nz, zb);
            if (iz >= 0) { *t = t1; return (uint32_t)ix + (uint32_t)iy * Nx + (uint32_t)iz * Nx * Ny + VAC_AND_OTH; }
        }
    }
    iz = -1;
    if ((p.z <= zb[0]) && (p.w > 0.0f)) { t1 = (zb[0] - p.z) / p.w; iz = 0; }
    else if ((p.z >= zb[Nz]) && (p.w < 0.0f)) { t1 = (zb[Nz] - p.z) / p.w; iz = (int)Nz - 1; }
    if ((iz >= 0) && (t1 <= *t)) {
        float x1 = p.x + p.u * t1;
        ix = isWhere(x1, Nx, xb);
        if (ix >= 0) {
            float y1 = p.y + p.v * t1;
            iy = isWhere(y1, Ny, yb);
            if (iy >= 0) { *t = t1; return (uint32_t)ix + (uint32_t)iy * Nx + (uint32_t)iz * Nx * Ny + VAC_AND_OTH; }
        }
    }
    return VACUUM_REG;
}

void hownear_phantom(ora_ctx *C, const ora_particle *p0, float *tperp)
{
    const gegs_scene *S = C->S;
    const float *xb = S->x_bounds, *yb = S->y_bounds, *zb = S->z_bounds;
    uint32_t Nx = (uint32_t)S->nx, Ny = (uint32_t)S->ny, Nz = (uint32_t)S->nz;
    ptr6 p = to_patient(C, p0);
    uint32_t off = (uint32_t)S->hownear_region_offset;
    *tperp = INFI_DIST;
    if (p0->region > off - 1u) {
        uint32_t ir = p0->region - off;
        int iz = (int)(ir / (Nx * Ny));
        ir -= (uint32_t)iz * Nx * Ny;
        int iy = (int)(ir / Nx);
        int ix = (int)(ir - (uint32_t)iy * Nx);
        float tx, ty, tz, tmp;
        tmp = xb[ix + 1] - p.x; tx = p.x - xb[ix]; if (tmp < tx) tx = tmp;
        tmp = yb[iy + 1] - p.y; ty = p.y - yb[iy]; if (tmp < ty) ty = tmp;
        /* with the reference decode (region - 5) the last voxel maps to iz = nz;
         * the plane past the end is taken as the last plane (the reference
         * reads one element past its z_bounds allocation there) */
        tmp = zb[(uint32_t)(iz + 1) <= Nz ? iz + 1 : (int)Nz] - p.z; tz = p.z - zb[iz]; if (tmp < tz) tz = tmp;
        if (tx < ty) *tperp = tx; else *tperp = ty;
        if (*tperp > tz) *tperp = tz;
    } else {
        float p1x = xb[0], p1y = yb[0], p1z = zb[0];
        float p2x = xb[Nx], p2y = yb[Ny], p2z = zb[Nz];
        if (p.x - p1x > 0 && p.x - p2x > 0) p2x = p2x; else if (p.x - p1x < 0 && p.x - p2x < 0) p2x = p1x; else p2x = p.x;
        if (p.y - p1y > 0 && p.y - p2y > 0) p2y = p2y; else if (p.y - p1y < 0 && p.y - p2y < 0) p2y = p1y; else p2y = p.y;
        if (p.z - p1z > 0 && p.z - p2z > 0) p2z = p2z; else if (p.z - p1z < 0 && p.z - p2z < 0) p2z = p1z; else p2z = p.z;
        *tperp = sqrtf((p.x - p2x) * (p.x - p2x) + (p.y - p2y) * (p.y - p2y) + (p.z - p2z) * (p.z - p2z));
    }
}

/* ---- polygons ----------------------------------------------------------- */
static int pointInPolygon(pt2 p, const float (*poly)[2], int n)
{
    int j = n - 1, odd = 0;
    for (int i = 0; i < n; i++) {
        float xi = poly[i][0], yi = poly[i][1], xj = poly[j][0], yj = poly[j][1];
        if (((yi < p.y && yj >= p.y) || (yj < p.y && yi >= p.y)) && (xi <= p.x || xj <= p.x))
            odd ^= (xi + (p.y - yi) / (yj - yi) * (xj - xi) < p.x);
        j = i;
    }
    return odd;
}

static int pointInLeaf(pt2 p, const float (*endn)[2])
{
    int bank = 0;
    if (pointInPolygon(p, endn, 17)) bank = 1;
    else if (pointInPolygon(p, endn + 17, 17)) bank = 2;
    return bank;
}

static int indexOfLeaf(const gegs_scene *S, pt2 p)
{
    int i = OUTMLC, index = OUTMLC;
    float x = p.x / p.y * S->mlc_zmin;
    float z = p.y - S->mlc_zmin;
    if (z < 0 || z > S->mlc_zthick) return index;
    if (x < S->mlc_x_start || x > S->mlc_x_end) return index;
    float wt = S->mlc_wt, gap = S->mlc_air_gap;
    if (x < S->mlc_x_start + wt) i = 0;
    else if (x < S->mlc_x_mid_1 + wt) i = (int)((x - S->mlc_x_start - wt) / (S->mlc_wl_full + gap));
    else if (x < S->mlc_x_mid_2 + wt) {
        i = (int)((x - S->mlc_x_mid_1 - wt) / (S->mlc_wl_target + S->mlc_wl_isocenter + gap * 2));
        if (x - S->mlc_x_mid_1 - wt - (S->mlc_wl_target + S->mlc_wl_isocenter + gap * 2) * (float)i < S->mlc_wl_target + gap)
            i = 10 + i * 2;
        else
            i = 11 + i * 2;
    } else if (x < S->mlc_x_end - S->mlc_wl_full)
        i = (int)((x - S->mlc_x_mid_2 - wt) / (S->mlc_wl_full + gap)) + 50;
    else if (x <= S->mlc_x_end)
        i = 58;
    if (i >= 0) {
        if (pointInPolygon(p, (const float (*)[2])S->crossXZ[i * 16], 14)) index = i;
        else if (i < 59) {
            if (pointInPolygon(p, (const float (*)[2])S->crossXZ[(i + 1) * 16], 14)) index = i + 1;
            else index = -(i + 1);
        } else index = OUTMLC;
    }
    return index;
}

static float rayIntersectPolygon(pt2 p0, pt2 v, const float (*poly)[2], int n, int *inside)
{
    float minDist = INFI_DIST + 1;
    int count = 0;
    for (int i = 0; i < n; i++) {
        float x1 = poly[i][0], y1 = poly[i][1];
        int j = i + 1;
        if (j >= n) j = 0;
        float x2 = poly[j][0], y2 = poly[j][1];
        float tmp1 = v.x * (y2 - y1) - v.y * (x2 - x1);
        if (tmp1 != 0) {
            float dist = ((x2 - x1) * (p0.y - y1) - (y2 - y1) * (p0.x - x1)) / tmp1;
            float u = ((x1 - p0.x) * v.y - (y1 - p0.y) * v.x) / tmp1;
            if (dist >= 0 && (u >= 0) && (u < 1)) {
                count++;
                if (dist < minDist) minDist = dist;
            }
        }
    }
    *inside = count & 1;
    return minDist;
}

static uint32_t inwhere_MLC(const gegs_scene *S, const gegs_field *F, float qx, float qy, float qz, int *index, int *Bank)
{
    uint32_t inew = DEFAULT_REG;
    pt2 p = {qx, qz};
    if (*index == OUTMLC) *index = indexOfLeaf(S, p);
    p.x = qy;
    if (*index >= 0) {
        *Bank = pointInLeaf(p, (const float (*)[2])F->endnode[*index]);
        if (*Bank > 0) inew = MLC_REGION; else inew = DEFAULT_REG;
    }
    return inew;
}

static uint32_t howfar_MLC(ora_ctx *C, ora_particle *p0, float *t)
{
    const gegs_scene *S = C->S;
    const gegs_field *F = &S->fields[p0->field];
    ora_particle p = *p0;
    uint32_t inew = p.region;
    int bank = p.bank;
    int index = p.leafIndex;
    int indexLimit1 = 0, indexLimit2 = 60;
    if (p.y < -S->mlc_rmax || p.y > S->mlc_rmax) return VACUUM_REG;
    float minDist, minBoundaryDist;
    float dis_xz, dis_yz, temp1 = INFI_DIST + 1;
    pt2 p1 = {p.x, p.z}, p2 = {p.y, p.z}, dir1 = {p.u, p.w}, dir2 = {p.v, p.w}, p3;
    int inside_XZ, inside_YZ;
    dis_xz = rayIntersectPolygon(p1, dir1, (const float (*)[2])S->boundaryXZ, 4, &inside_XZ);
    dis_yz = rayIntersectPolygon(p2, dir2, (const float (*)[2])S->boundaryYZ, 4, &inside_YZ);
    if (dis_xz >= INFI_DIST || dis_yz >= INFI_DIST) return VACUUM_REG;
    if (dis_xz < dis_yz) minBoundaryDist = dis_xz; else minBoundaryDist = dis_yz;
    if (inside_XZ && inside_YZ) {
        p3.x = p1.x + dis_xz * dir1.x;
        p3.y = p1.y + (dis_xz - 0.001) * dir1.y;
        indexLimit1 = indexOfLeaf(S, p3);
        if (indexLimit1 < 0) indexLimit1 = -indexLimit1;
    } else {
        inew = VACUUM_REG;
        if (minBoundaryDist >= INFI_DIST) return inew;
        if (*t > minBoundaryDist) {
            *t = minBoundaryDist + EPSTEP;
            goto NewRegion;
        }
        return inew;
    }
    if (p.leafIndex > -60) index = p.leafIndex;
    else index = indexOfLeaf(S, p1);
    if (index >= 0) {
        dis_xz = rayIntersectPolygon(p1, dir1, (const float (*)[2])S->crossXZ[index * 16], 14, &inside_XZ);
        const float (*yzp)[2] = (const float (*)[2])F->endnode[index];
        int nv = 17;
        switch (p.bank) {
        case 0: yzp = (const float (*)[2])F->endnode[index][2]; nv = 30; break;
        case 2: yzp = (const float (*)[2])F->endnode[index][17]; break;
        }
        dis_yz = rayIntersectPolygon(p2, dir2, yzp, nv, &inside_YZ);
        if (dis_yz > dis_xz) {
            if (dir1.x < 0 && index > 0) index = -index;
            else if (index < 59) index = -(index + 1);
        }
    } else if (index > -60) {
        int sx = 1, sl = 16;
        if (dir1.x < 0) { sx = -1; sl = -16; if (indexLimit1 > 0) indexLimit1 -= 1; indexLimit2 = -index + 1; }
        else { indexLimit2 = indexLimit1; indexLimit1 = -index - 1; }
        int i = -index - sx;
        if (indexLimit1 < 0) indexLimit1 = 0;
        if (indexLimit2 > 59) indexLimit2 = 59;
        if (i < 0) i = 0;
        if (i > 59) i = 59;
        int lp = i * 16;
        do {
            temp1 = rayIntersectPolygon(p1, dir1, (const float (*)[2])S->crossXZ[lp], 14, &inside_XZ);
            i += sx;
            lp += sl;
        } while (i >= indexLimit1 && i <= indexLimit2 && temp1 >= INFI_DIST);
        if (temp1 < dis_xz) {
            dis_xz = temp1;
            index = i - sx;
        } else {
            index = PASSMLC;
            p0->module = (uint8_t)S->module_order[GEGS_M_VARMLC];
        }
    }
    if (dis_xz < dis_yz) minDist = dis_xz; else minDist = dis_yz;
    {
        int steppingOut = 0;
        if ((minDist + EPSTEP) >= minBoundaryDist) { minDist = minBoundaryDist; steppingOut = 1; }
        if (*t > minDist) {
            *t = minDist + EPSTEP;
            if (steppingOut) {
                inew = DEFAULT_REG;
                p0->leafIndex = PASSMLC;
                p0->module = (uint8_t)S->module_order[GEGS_M_VARMLC];
                return inew;
            }
        } else return inew;
    }
NewRegion:
    {
        float qx = p.x + *t * p.u, qy = p.y + *t * p.v, qz = p.z + *t * p.w;
        inew = inwhere_MLC(S, F, qx, qy, qz, &index, &bank);
        p0->leafIndex = (int8_t)index;
        p0->bank = (int8_t)bank;
    }
    return inew;
}

/* jaws: ROTATE_SecJaws_XY is defined in the reference (CUDA_EGS.h:24) */
static uint32_t howfar_SecJawsY(ora_ctx *C, ora_particle *p, float *t)
{
    const gegs_scene *S = C->S;
    const gegs_field *F = &S->fields[p->field];
    uint32_t inew = VACUUM_REG;
    pt2 p0, p1 = {p->y, p->z}, p2 = {p->x, p->z}, dir1 = {p->v, p->w}, dir2 = {p->u, p->w};
    int inside_XZ, inside_YZ;
    float dis_xz = rayIntersectPolygon(p1, dir1, (const float (*)[2])F->boundMaxY, 4, &inside_XZ);
    float dis_yz = rayIntersectPolygon(p2, dir2, (const float (*)[2])F->boundMaxY, 4, &inside_YZ);
    float minBoundaryDist;
    if (dis_xz >= INFI_DIST || dis_yz >= INFI_DIST) return inew;
    if (dis_xz < dis_yz) minBoundaryDist = dis_xz; else minBoundaryDist = dis_yz;
    if (inside_XZ && inside_YZ) {
        if (pointInPolygon(p2, (const float (*)[2])F->jawsGeomY[2], 4)) {
            inew = DEFAULT_REG;
            dis_xz = rayIntersectPolygon(p2, dir2, (const float (*)[2])F->jawsGeomY, 4, &inside_YZ);
            dis_yz = rayIntersectPolygon(p2, dir2, (const float (*)[2])F->jawsGeomY[4], 4, &inside_YZ);
            if (dis_xz < INFI_DIST) {
                if (*t > dis_xz) { inew = SECJAWS_REG; *t = dis_xz + EPSTEP; }
            } else if (dis_yz < INFI_DIST) {
                if (*t > dis_yz) { inew = SECJAWS_REG; *t = dis_yz + EPSTEP; }
            } else {
                if (*t > minBoundaryDist) { *t = minBoundaryDist + EPSTEP; p->module = (uint8_t)S->module_order[GEGS_M_SECJAWY]; }
            }
        } else {
            inew = SECJAWS_REG;
            dis_yz = rayIntersectPolygon(p2, dir2, (const float (*)[2])F->jawsGeomY[2], 4, &inside_YZ);
            if (dis_yz < INFI_DIST) {
                if (*t > dis_yz) { inew = DEFAULT_REG; *t = dis_yz + EPSTEP; }
            } else {
                if (*t > minBoundaryDist) { inew = VACUUM_REG; *t = minBoundaryDist + EPSTEP; }
            }
        }
    } else {
        inew = DEFAULT_REG;
        if (*t > minBoundaryDist) {
            *t = minBoundaryDist + EPSTEP;
            p0.x = p->y + *t * p->v;
            p0.y = p->x + *t * p->u;
            if (!pointInPolygon(p0, (const float (*)[2])F->boundMinY, 4)) inew = VACUUM_REG;
            else {
                p0.x = p0.y;
                p0.y = p->z + *t * p->w;
                if (pointInPolygon(p0, (const float (*)[2])F->jawsGeomY[2], 4)) inew = DEFAULT_REG;
                else inew = SECJAWS_REG;
            }
        }
    }
    return inew;
}

static uint32_t howfar_SecJawsX(ora_ctx *C, ora_particle *p, float *t)
{
    const gegs_scene *S = C->S;
    const gegs_field *F = &S->fields[p->field];
    uint32_t inew = VACUUM_REG;
    pt2 p0, p1 = {p->y, p->z}, p2 = {p->x, p->z}, dir1 = {p->v, p->w}, dir2 = {p->u, p->w};
    int inside_XZ, inside_YZ;
    float dis_xz = rayIntersectPolygon(p1, dir1, (const float (*)[2])F->boundMaxX, 4, &inside_XZ);
    float dis_yz = rayIntersectPolygon(p2, dir2, (const float (*)[2])F->boundMaxX, 4, &inside_YZ);
    float minBoundaryDist;
    if (dis_xz >= INFI_DIST || dis_yz >= INFI_DIST) return inew;
    if (dis_xz < dis_yz) minBoundaryDist = dis_xz; else minBoundaryDist = dis_yz;
    if (inside_XZ && inside_YZ) {
        if (pointInPolygon(p1, (const float (*)[2])F->jawsGeomX[2], 4)) {
            inew = DEFAULT_REG;
            dis_xz = rayIntersectPolygon(p1, dir1, (const float (*)[2])F->jawsGeomX, 4, &inside_XZ);
            dis_yz = rayIntersectPolygon(p1, dir1, (const float (*)[2])F->jawsGeomX[4], 4, &inside_XZ);
            if (dis_xz < INFI_DIST) {
                if (*t > dis_xz) { inew = SECJAWS_REG; *t = dis_xz + EPSTEP; }
            } else if (dis_yz < INFI_DIST) {
                if (*t > dis_yz) { inew = SECJAWS_REG; *t = dis_yz + EPSTEP; }
            } else {
                if (*t > minBoundaryDist) { *t = minBoundaryDist + EPSTEP; p->module = (uint8_t)S->module_order[GEGS_M_SECJAWX]; }
            }
        } else {
            inew = SECJAWS_REG;
            dis_xz = rayIntersectPolygon(p1, dir1, (const float (*)[2])F->jawsGeomX[2], 4, &inside_XZ);
            if (dis_xz < INFI_DIST) {
                if (*t > dis_xz) { inew = DEFAULT_REG; *t = dis_yz + EPSTEP; }
            } else {
                if (*t > minBoundaryDist) { inew = VACUUM_REG; *t = minBoundaryDist + EPSTEP; }
            }
        }
    } else {
        inew = DEFAULT_REG;
        if (*t > minBoundaryDist) {
            *t = minBoundaryDist + EPSTEP;
            p0.x = p->y + *t * p->v;
            p0.y = p->x + *t * p->u;
            if (!pointInPolygon(p0, (const float (*)[2])F->boundMinX, 4)) inew = VACUUM_REG;
            else {
                p0.y = p->z + *t * p->w;
                if (pointInPolygon(p0, (const float (*)[2])F->jawsGeomX[2], 4)) inew = DEFAULT_REG;
                else inew = SECJAWS_REG;
            }
        }
    }
    return inew;
}

/* ---- hownear ------------------------------------------------------------ */
static float dist2p(pt2 v, pt2 w) { return (v.x - w.x) * (v.x - w.x) + (v.y - w.y) * (v.y - w.y); }
static float distp(pt2 v, pt2 w) { return sqrtf((v.x - w.x) * (v.x - w.x) + (v.y - w.y) * (v.y - w.y)); }

static float pointDistToSegment(pt2 p, pt2 v, pt2 w)
{
    float l2 = dist2p(v, w);
    if (l2 == 0) return distp(p, v);
    float t = ((p.x - v.x) * (w.x - v.x) + (p.y - v.y) * (w.y - v.y)) / l2;
    if (t < 0) return distp(p, v);
    if (t > 1) return distp(p, w);
    pt2 a = {v.x + t * (w.x - v.x), v.y + t * (w.y - v.y)};
    return distp(p, a);
}

static float pointMinDistToPolygon(pt2 p0, const float (*poly)[2], int n)
{
    float minDist = 1e9;
    for (int i = 0; i < n; i++) {
        int j = i + 1;
        if (j >= n) j = 0;
        float d = pointDistToSegment(p0, P2(poly[i]), P2(poly[j]));
        if (d < minDist) minDist = d;
    }
    return minDist;
}

static void hownear_MLC(ora_ctx *C, ora_particle *p, float *tperp)
{
    const gegs_scene *S = C->S;
    const gegs_field *F = &S->fields[p->field];
    pt2 p1 = {p->x, p->z}, p2 = {p->y, p->z};
    int index;
    float tperp_xz = INFI_DIST + 1, tperp_yz = INFI_DIST + 1, bound;
    int inside_XZ, inside_YZ;
    if (p->leafIndex < -60) {
        inside_XZ = pointInPolygon(p1, (const float (*)[2])S->boundaryXZ, 4);
        inside_YZ = pointInPolygon(p2, (const float (*)[2])S->boundaryYZ, 4);
    } else { inside_XZ = 1; inside_YZ = 1; }
    float bxz = pointMinDistToPolygon(p1, (const float (*)[2])S->boundaryXZ, 4);
    float byz = pointMinDistToPolygon(p2, (const float (*)[2])S->boundaryYZ, 4);
    if (bxz < byz) bound = bxz; else bound = byz;
    if (inside_XZ && inside_YZ) {
        if (p->leafIndex > PASSMLC) index = p->leafIndex;
        else { index = indexOfLeaf(S, p1); p->leafIndex = (int8_t)index; }
        if (index >= 0) {
            tperp_xz = pointMinDistToPolygon(p1, (const float (*)[2])S->crossXZ[index * 16], 14);
            if (p->bank < 0) p->bank = (int8_t)pointInLeaf(p2, (const float (*)[2])F->endnode[index]);
            const float (*yzp)[2] = (const float (*)[2])F->endnode[index];
            int nv = 17;
            switch (p->bank) {
            case 0: yzp = (const float (*)[2])F->endnode[index][2]; nv = 30; break;
            case 2: yzp = (const float (*)[2])F->endnode[index][17]; break;
            }
            tperp_yz = pointMinDistToPolygon(p2, yzp, nv);
        } else if (index > -60) {
            int i = -index;
            float t1 = pointMinDistToPolygon(p1, (const float (*)[2])S->crossXZ[i * 16], 14);
            i--;
            tperp_xz = pointMinDistToPolygon(p1, (const float (*)[2])S->crossXZ[i * 16], 14);
            if (t1 < tperp_xz) tperp_xz = t1;
        }
        if (tperp_xz < tperp_yz) *tperp = tperp_xz; else *tperp = tperp_yz;
    } else {
        *tperp = bound;
    }
}

static void hownear_SecJawsY(ora_ctx *C, ora_particle *p, float *tperp)
{
    const gegs_field *F = &C->S->fields[p->field];
    pt2 p1 = {p->y, p->z}, p2 = {p->x, p->z};
    int inside_XZ = pointInPolygon(p1, (const float (*)[2])F->boundMaxY, 4);
    int inside_YZ = pointInPolygon(p2, (const float (*)[2])F->boundMaxY, 4);
    float bound_xz = pointMinDistToPolygon(p1, (const float (*)[2])F->boundMaxY, 4);
    float bound_yz = pointMinDistToPolygon(p2, (const float (*)[2])F->boundMaxY, 4);
    if (inside_XZ && inside_YZ) {
        float dist_yz = pointMinDistToPolygon(p2, (const float (*)[2])F->jawsGeomY[2], 4);
        if (pointInPolygon(p2, (const float (*)[2])F->jawsGeomY[2], 4)) {
            if (dist_yz < bound_xz) *tperp = dist_yz; else *tperp = bound_xz;
        } else {
            if (dist_yz > bound_yz) dist_yz = bound_yz;
            if (dist_yz < bound_xz) *tperp = dist_yz; else *tperp = bound_xz;
        }
    } else {
        if (bound_xz < bound_yz) *tperp = bound_xz; else *tperp = bound_yz;
    }
}

static void hownear_SecJawsX(ora_ctx *C, ora_particle *p, float *tperp)
{
    const gegs_field *F = &C->S->fields[p->field];
    pt2 p1 = {p->y, p->z}, p2 = {p->x, p->z};
    int inside_XZ = pointInPolygon(p1, (const float (*)[2])F->boundMaxX, 4);
    int inside_YZ = pointInPolygon(p2, (const float (*)[2])F->boundMaxX, 4);
    float bound_xz = pointMinDistToPolygon(p1, (const float (*)[2])F->boundMaxX, 4);
    float bound_yz = pointMinDistToPolygon(p2, (const float (*)[2])F->boundMaxX, 4);
    if (inside_XZ && inside_YZ) {
        float dist_xz = pointMinDistToPolygon(p1, (const float (*)[2])F->jawsGeomX[2], 4);
        if (pointInPolygon(p1, (const float (*)[2])F->jawsGeomX[2], 4)) {
            if (dist_xz < bound_yz) *tperp = dist_xz; else *tperp = bound_yz;
        } else {
            if (dist_xz > bound_xz) dist_xz = bound_xz;
            if (dist_xz < bound_yz) *tperp = dist_xz; else *tperp = bound_yz;
        }
    } else {
        if (bound_xz < bound_yz) *tperp = bound_xz; else *tperp = bound_yz;
    }
}

/* ---- dispatch on the particle's module (photon.cu:142-158) --------------- */
uint32_t ora_howfar(ora_ctx *C, ora_particle *p, float *t, int *ok)
{
    *ok = 1;
    switch (p->module) {
    case GEGS_M_SECJAWY: return howfar_SecJawsY(C, p, t);
    case GEGS_M_SECJAWX: return howfar_SecJawsX(C, p, t);
    case GEGS_M_VARMLC: return howfar_MLC(C, p, t);
    case GEGS_M_PHANTOM: return howfar_phantom(C, p, t);
    default: *ok = 0; return 0;
    }
}

void ora_hownear(ora_ctx *C, ora_particle *p, float *tperp, int *ok)
{
    *ok = 1;
    switch (p->module) {
    case GEGS_M_SECJAWY: hownear_SecJawsY(C, p, tperp); return;
    case GEGS_M_SECJAWX: hownear_SecJawsX(C, p, tperp); return;
    case GEGS_M_VARMLC: hownear_MLC(C, p, tperp); return;
    case GEGS_M_PHANTOM: hownear_phantom(C, p, tperp); return;
    default: *ok = 0; *tperp = 0; return;
    }
}
