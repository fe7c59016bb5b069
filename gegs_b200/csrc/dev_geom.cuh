// Device geometry: beam->patient transform and one-plane voxel DDA
// (howfar_phantom, geom.cu:54-307), isotropic distance to the voxel walls
// (hownear_phantom, geom.cu:1422-1543), DYNVMLC leaf tracking (howfar_MLC /
// hownear_MLC, geom.cu:310-790, 1152-1286) and the secondary jaws
// (geom.cu:793-1035, 1288-1374).  The reference's behaviour is kept, including
// its hownear voxel decode (region - 5, selectable) and the dis_yz step of
// howfar_SecJawsX inside the tungsten.
#pragma once
#include "dev_common.cuh"

struct P6 { float x, y, z, u, v, w; };

__device__ __forceinline__ P6 to_patient(const DevCtx &C, const Part &p0)
{
    const gegs_field *F = &C.fields[p0.field];
    float ca = __ldg(&F->cos_angle), sa = __ldg(&F->sin_angle);
    P6 p;
    if (C.change_xyz) {
        p.x = p0.y; p.y = p0.z - C.sid; p.z = p0.x;
        p.u = p0.v; p.v = p0.w; p.w = p0.u;
    } else {
        p.x = p0.x; p.y = p0.y; p.z = p0.z - C.sid;
        p.u = p0.u; p.v = p0.v; p.w = p0.w;
    }
    float tx = p.x * ca - p.y * sa;
    float ty = p.x * sa + p.y * ca;
    p.x = tx; p.y = ty;
    tx = p.u * ca - p.v * sa;
    ty = p.u * sa + p.v * ca;
    p.u = tx; p.v = ty;
    p.x = p.x + C.iso0;
    p.y = p.y + C.iso1;
    p.z = p.z + C.iso2;
    return p;
}

__device__ __forceinline__ int is_where(float p, uint32_t nreg, const float *bounds)
{
    if ((p < __ldg(&bounds[0])) || (p > __ldg(&bounds[nreg]))) return -1;
    if (nreg == 1) return 0;
    int ml = 0, mu = (int)nreg;
    while (mu - ml > 1) {
        int mav = (ml + mu) / 2;
        if (p <= __ldg(&bounds[mav])) mu = mav; else ml = mav;
    }
    return mu - 1;
}

__device__ uint32_t howfar_phantom(const DevCtx &C, const Part &p0, float &t)
{
    const float *xb = C.xb, *yb = C.yb, *zb = C.zb;
    uint32_t Nx = (uint32_t)C.nx, Ny = (uint32_t)C.ny, Nz = (uint32_t)C.nz;
    P6 p = to_patient(C, p0);
    uint32_t region = p0.region;
    if (region >= GX_VAC_AND_OTH) {
        uint32_t ir = region - GX_VAC_AND_OTH;
        int iz = (int)fastdiv(C.div_nxny, ir);
        ir -= (uint32_t)iz * Nx * Ny;
        int iy = (int)fastdiv(C.div_nx, ir);
        int ix = (int)(ir - (uint32_t)iy * Nx);
        uint32_t inew = region;
        if (p.u > 0.0f) {
            float d = (__ldg(&xb[ix + 1]) - p.x) / p.u;
            if (d <= t) { t = d; if ((uint32_t)(++ix) < Nx) inew = region + 1; else inew = 0; }
        } else if (p.u < 0.0f) {
            float d = (__ldg(&xb[ix]) - p.x) / p.u;
            if (d <= t) { t = d; if (--ix >= 0) inew = region - 1; else inew = 0; }
        }
        if (p.v > 0.0f) {
            float d = (__ldg(&yb[iy + 1]) - p.y) / p.v;
            if (d <= t) { t = d; if ((uint32_t)(++iy) < Ny) inew = region + Nx; else inew = 0; }
        } else if (p.v < 0.0f) {
            float d = (__ldg(&yb[iy]) - p.y) / p.v;
            if (d <= t) { t = d; if (--iy >= 0) inew = region - Nx; else inew = 0; }
        }
        if (p.w > 0.0f) {
            float d = (__ldg(&zb[iz + 1]) - p.z) / p.w;
            if (d <= t) { t = d; if ((uint32_t)(++iz) < Nz) inew = region + Nx * Ny; else inew = 0; }
        } else if (p.w < 0.0f) {
            float d = (__ldg(&zb[iz]) - p.z) / p.w;
            if (d <= t) { t = d; if (--iz >= 0) inew = region - Nx * Ny; else inew = 0; }
        }
        if (t < 0) t = GX_EPSTEP;
        return inew;
    }
    int ix, iy, iz;
    float t1 = 0.0f;
    ix = -1;
    if ((p.x <= __ldg(&xb[0])) && (p.u > 0.0f)) { t1 = (__ldg(&xb[0]) - p.x) / p.u; ix = 0; }
    else if ((p.x >= __ldg(&xb[Nx])) && (p.u < 0.0f)) { t1 = (__ldg(&xb[Nx]) - p.x) / p.u; ix = (int)Nx - 1; }
    if ((ix >= 0) && (t1 <= t)) {
        float y1 = p.y + p.v * t1;
        iy = is_where(y1, Ny, yb);
        if (iy >= 0) {
            float z1 = p.z + p.w * t1;
            iz = is_where(z1, Nz, zb);
            if (iz >= 0) { t = t1; return (uint32_t)ix + (uint32_t)iy * Nx + (uint32_t)iz * Nx * Ny + GX_VAC_AND_OTH; }
        }
    }
    iy = -1;
    if ((p.y <= __ldg(&yb[0])) && (p.v > 0.0f)) { t1 = (__ldg(&yb[0]) - p.y) / p.v; iy = 0; }
    else if ((p.y >= __ldg(&yb[Ny])) && (p.v < 0.0f)) { t1 = (__ldg(&yb[Ny]) - p.y) / p.v; iy = (int)Ny - 1; }
    if ((iy >= 0) && (t1 <= t)) {
        float x1 = p.x + p.u * t1;
        ix = is_where(x1, Nx, xb);
        if (ix >= 0) {
            float z1 = p.z + p.w * t1;
            iz = is_where(z1, Nz, zb);
            if (iz >= 0) { t = t1; return (uint32_t)ix + (uint32_t)iy * Nx + (uint32_t)iz * Nx * Ny + GX_VAC_AND_OTH; }
        }
    }
    iz = -1;
    if ((p.z <= __ldg(&zb[0])) && (p.w > 0.0f)) { t1 = (__ldg(&zb[0]) - p.z) / p.w; iz = 0; }
    else if ((p.z >= __ldg(&zb[Nz])) && (p.w < 0.0f)) { t1 = (__ldg(&zb[Nz]) - p.z) / p.w; iz = (int)Nz - 1; }
    if ((iz >= 0) && (t1 <= t)) {
        float x1 = p.x + p.u * t1;
        ix = is_where(x1, Nx, xb);
        if (ix >= 0) {
            float y1 = p.y + p.v * t1;
            iy = is_where(y1, Ny, yb);
            if (iy >= 0) { t = t1; return (uint32_t)ix + (uint32_t)iy * Nx + (uint32_t)iz * Nx * Ny + GX_VAC_AND_OTH; }
        }
    }
    return 0;
}

__device__ void hownear_phantom(const DevCtx &C, const Part &p0, float &tperp)
{
    const float *xb = C.xb, *yb = C.yb, *zb = C.zb;
    uint32_t Nx = (uint32_t)C.nx, Ny = (uint32_t)C.ny, Nz = (uint32_t)C.nz;
    P6 p = to_patient(C, p0);
    uint32_t off = (uint32_t)C.hownear_off;
    tperp = GX_INFI_DIST;
    if (p0.region > off - 1u) {
        uint32_t ir = p0.region - off;
        int iz = (int)fastdiv(C.div_nxny, ir);
        ir -= (uint32_t)iz * Nx * Ny;
        int iy = (int)fastdiv(C.div_nx, ir);
        int ix = (int)(ir - (uint32_t)iy * Nx);
        float tx, ty, tz, tmp;
        tmp = __ldg(&xb[ix + 1]) - p.x; tx = p.x - __ldg(&xb[ix]); if (tmp < tx) tx = tmp;
        tmp = __ldg(&yb[iy + 1]) - p.y; ty = p.y - __ldg(&yb[iy]); if (tmp < ty) ty = tmp;
        // the reference decode maps the last voxel to iz = nz: the missing plane is the last plane
        tmp = __ldg(&zb[(uint32_t)(iz + 1) <= Nz ? iz + 1 : (int)Nz]) - p.z; tz = p.z - __ldg(&zb[iz]); if (tmp < tz) tz = tmp;
        if (tx < ty) tperp = tx; else tperp = ty;
        if (tperp > tz) tperp = tz;
    } else {
        float p1x = __ldg(&xb[0]), p1y = __ldg(&yb[0]), p1z = __ldg(&zb[0]);
        float p2x = __ldg(&xb[Nx]), p2y = __ldg(&yb[Ny]), p2z = __ldg(&zb[Nz]);
        if (p.x - p1x > 0 && p.x - p2x > 0) {} else if (p.x - p1x < 0 && p.x - p2x < 0) p2x = p1x; else p2x = p.x;
        if (p.y - p1y > 0 && p.y - p2y > 0) {} else if (p.y - p1y < 0 && p.y - p2y < 0) p2y = p1y; else p2y = p.y;
        if (p.z - p1z > 0 && p.z - p2z > 0) {} else if (p.z - p1z < 0 && p.z - p2z < 0) p2z = p1z; else p2z = p.z;
        tperp = sqrtf((p.x - p2x) * (p.x - p2x) + (p.y - p2y) * (p.y - p2y) + (p.z - p2z) * (p.z - p2z));
    }
}

// ---- polygons (2-D points as float2) ----------------------------------------
__device__ __forceinline__ float2 ld2(const float2 *a) { return __ldg(a); }

__device__ int point_in_polygon(float2 p, const float2 *poly, int n)
{
    int j = n - 1, odd = 0;
    for (int i = 0; i < n; i++) {
        float2 a = ld2(&poly[i]), b = ld2(&poly[j]);
        if (((a.y < p.y && b.y >= p.y) || (b.y < p.y && a.y >= p.y)) && (a.x <= p.x || b.x <= p.x))
            odd ^= (a.x + (p.y - a.y) / (b.y - a.y) * (b.x - a.x) < p.x);
        j = i;
    }
    return odd;
}

__device__ int point_in_polygon_local(float2 p, const float2 *poly, int n)
{
    int j = n - 1, odd = 0;
    for (int i = 0; i < n; i++) {
        float2 a = poly[i], b = poly[j];
        if (((a.y < p.y && b.y >= p.y) || (b.y < p.y && a.y >= p.y)) && (a.x <= p.x || b.x <= p.x))
            odd ^= (a.x + (p.y - a.y) / (b.y - a.y) * (b.x - a.x) < p.x);
        j = i;
    }
    return odd;
}

__device__ __forceinline__ const float2 *endnode_of(const DevCtx &C, int field, int leaf)
{
    return reinterpret_cast<const float2 *>(&C.fields[field].endnode[leaf][0][0]);
}

__device__ int point_in_leaf(float2 p, const float2 *endn)
{
    int bank = 0;
    if (point_in_polygon(p, endn, 17)) bank = 1;
    else if (point_in_polygon(p, endn + 17, 17)) bank = 2;
    return bank;
}

__device__ int index_of_leaf(const DevCtx &C, float2 p)
{
    int i = GX_OUTMLC, index = GX_OUTMLC;
    float x = p.x / p.y * C.mlc_zmin;
    float z = p.y - C.mlc_zmin;
    if (z < 0 || z > C.mlc_zthick) return index;
    if (x < C.mlc_x_start || x > C.mlc_x_end) return index;
    float wt = C.mlc_wt, gap = C.mlc_air_gap;
    if (x < C.mlc_x_start + wt) i = 0;
    else if (x < C.mlc_x_mid_1 + wt) i = (int)((x - C.mlc_x_start - wt) / (C.mlc_wl_full + gap));
    else if (x < C.mlc_x_mid_2 + wt) {
        i = (int)((x - C.mlc_x_mid_1 - wt) / (C.mlc_wl_target + C.mlc_wl_isocenter + gap * 2));
        if (x - C.mlc_x_mid_1 - wt - (C.mlc_wl_target + C.mlc_wl_isocenter + gap * 2) * (float)i < C.mlc_wl_target + gap)
            i = 10 + i * 2;
        else
            i = 11 + i * 2;
    } else if (x < C.mlc_x_end - C.mlc_wl_full)
        i = (int)((x - C.mlc_x_mid_2 - wt) / (C.mlc_wl_full + gap)) + 50;
    else if (x <= C.mlc_x_end)
        i = 58;
    if (i >= 0) {
        if (point_in_polygon(p, C.crossXZ + i * 16, 14)) index = i;
        else if (i < 59) {
            if (point_in_polygon(p, C.crossXZ + (i + 1) * 16, 14)) index = i + 1;
            else index = -(i + 1);
        } else index = GX_OUTMLC;
    }
    return index;
}

// (u >= 0 && u < 1) for u = fl(num / den), den != 0, deciding from num and
// den without the division where the outcome is certain and dividing
// otherwise, so the decision is always that of the rounded quotient:
// with n = num * sign(den) and d = |den| (exact), fl(num / den) = fl(n / d);
// n < -d * 1e-30 gives a negative quotient that does not round to zero; n >= d
// a quotient >= 1; 0 <= n <= d * (1 - 2^-20) a quotient below 1 - 2^-21.
__device__ __forceinline__ bool edge_param_in_unit(float num, float den)
{
    float n = den > 0.0f ? num : -num;
    float d = fabsf(den);
    if (n < -d * 1e-30f) return false;
    if (n >= d) return false;
    if (n >= 0.0f && n <= d * 0.99999904632568359375f) return true;
    float u = num / den;
    return (u >= 0) && (u < 1);
}

template <bool LOCAL>
__device__ float ray_intersect_polygon(float2 p0, float2 v, const float2 *poly, int n, int &inside)
{
    float minDist = GX_INFI_DIST + 1;
    int count = 0;
    for (int i = 0; i < n; i++) {
        int j = i + 1;
        if (j >= n) j = 0;
        float2 a = LOCAL ? poly[i] : ld2(&poly[i]);
        float2 b = LOCAL ? poly[j] : ld2(&poly[j]);
        float tmp1 = v.x * (b.y - a.y) - v.y * (b.x - a.x);
        if (tmp1 != 0) {
            // the edge parameter first: most edges fail it, and then the distance is not needed
            if (edge_param_in_unit(((a.x - p0.x) * v.y - (a.y - p0.y) * v.x), tmp1)) {
                float dist = ((b.x - a.x) * (p0.y - a.y) - (b.y - a.y) * (p0.x - a.x)) / tmp1;
                if (dist >= 0) {
                    count++;
                    if (dist < minDist) minDist = dist;
                }
            }
        }
    }
    inside = count & 1;
    return minDist;
}

__device__ uint32_t inwhere_mlc(const DevCtx &C, int field, float qx, float qy, float qz, int &index, int &bank)
{
    uint32_t inew = 1;
    float2 p = make_float2(qx, qz);
    if (index == GX_OUTMLC) index = index_of_leaf(C, p);
    p.x = qy;
    if (index >= 0) {
        bank = point_in_leaf(p, endnode_of(C, field, index));
        if (bank > 0) inew = 3; else inew = 1;
    }
    return inew;
}

__device__ uint32_t howfar_mlc(const DevCtx &C, Part &p0, float &t)
{
    const Part p = p0;
    uint32_t inew = p.region;
    int bank = p.bank;
    int index = p.leafIndex;
    int indexLimit1 = 0, indexLimit2 = 60;
    if (p.y < -C.mlc_rmax || p.y > C.mlc_rmax) return 0;
    float minDist, minBoundaryDist;
    float dis_xz, dis_yz, temp1 = GX_INFI_DIST + 1;
    float2 p1 = make_float2(p.x, p.z), p2 = make_float2(p.y, p.z);
    float2 dir1 = make_float2(p.u, p.w), dir2 = make_float2(p.v, p.w), p3;
    int inside_XZ, inside_YZ;
    dis_xz = ray_intersect_polygon<true>(p1, dir1, C.boundaryXZ, 4, inside_XZ);
    dis_yz = ray_intersect_polygon<true>(p2, dir2, C.boundaryYZ, 4, inside_YZ);
    if (dis_xz >= GX_INFI_DIST || dis_yz >= GX_INFI_DIST) return 0;
    if (dis_xz < dis_yz) minBoundaryDist = dis_xz; else minBoundaryDist = dis_yz;
    bool to_new_region = false;
    if (inside_XZ && inside_YZ) {
        p3.x = p1.x + dis_xz * dir1.x;
        p3.y = p1.y + (dis_xz - 0.001) * dir1.y;   // in double, as geom.cu:591
        indexLimit1 = index_of_leaf(C, p3);
        if (indexLimit1 < 0) indexLimit1 = -indexLimit1;
    } else {
        inew = 0;
        if (minBoundaryDist >= GX_INFI_DIST) return inew;
        if (t > minBoundaryDist) { t = minBoundaryDist + GX_EPSTEP; to_new_region = true; }
        else return inew;
    }
    if (!to_new_region) {
        if (p.leafIndex > -60) index = p.leafIndex;
        else index = index_of_leaf(C, p1);
        // In a leaf: the ray against the leaf's XZ cross section, then against
        // its YZ leaf-end outline. In an air gap: against the XZ cross sections
        // of the leaves the ray walks through, from the nearest, until one is
        // hit or the walk leaves the limits. One loop serves both, one polygon
        // per pass, so leaf and gap lanes of a warp intersect together (each
        // lane keeps the reference's polygons, points and order).
        if (index > -60) {
            const bool leaf = index >= 0;
            const float2 *yzp = nullptr;
            int nv = 17, sx = 1, sl = 16, i = 0, lp = 0;
            if (leaf) {
                yzp = endnode_of(C, p.field, index);
                if (p.bank == 0) { yzp += 2; nv = 30; }
                else if (p.bank == 2) { yzp += 17; }
            } else {
                if (dir1.x < 0) { sx = -1; sl = -16; if (indexLimit1 > 0) indexLimit1 -= 1; indexLimit2 = -index + 1; }
                else { indexLimit2 = indexLimit1; indexLimit1 = -index - 1; }
                i = -index - sx;
                if (indexLimit1 < 0) indexLimit1 = 0;
                if (indexLimit2 > 59) indexLimit2 = 59;
                if (i < 0) i = 0;
                if (i > 59) i = 59;
                lp = i * 16;
            }
            float leaf_xz = 0.0f, leaf_yz = 0.0f;
            int ins, pass = 0;
            bool more = true;
            while (more) {
                const bool yz = leaf && pass == 1;
                const float2 *poly = leaf ? (pass == 0 ? C.crossXZ + index * 16 : yzp) : C.crossXZ + lp;
                float d = ray_intersect_polygon<false>(yz ? p2 : p1, yz ? dir2 : dir1, poly, yz ? nv : 14, ins);
                if (leaf) {
                    if (pass == 0) leaf_xz = d;
                    else { leaf_yz = d; more = false; }
                } else {
                    temp1 = d;
                    i += sx;
                    lp += sl;
                    more = i >= indexLimit1 && i <= indexLimit2 && temp1 >= GX_INFI_DIST;
                }
                pass++;
            }
            if (leaf) {
                dis_xz = leaf_xz;
                dis_yz = leaf_yz;
                if (dis_yz > dis_xz) {
                    if (dir1.x < 0 && index > 0) index = -index;
                    else if (index < 59) index = -(index + 1);
                }
            } else if (temp1 < dis_xz) {
                dis_xz = temp1;
                index = i - sx;
            } else {
                index = GX_PASSMLC;
                p0.module = (uint8_t)C.module_order[GEGS_M_VARMLC];
            }
        }
        if (dis_xz < dis_yz) minDist = dis_xz; else minDist = dis_yz;
        bool steppingOut = false;
        if ((minDist + GX_EPSTEP) >= minBoundaryDist) { minDist = minBoundaryDist; steppingOut = true; }
        if (t > minDist) {
            t = minDist + GX_EPSTEP;
            if (steppingOut) {
                p0.leafIndex = GX_PASSMLC;
                p0.module = (uint8_t)C.module_order[GEGS_M_VARMLC];
                return 1;
            }
        } else return inew;
    }
    float qx = p.x + t * p.u, qy = p.y + t * p.v, qz = p.z + t * p.w;
    inew = inwhere_mlc(C, p.field, qx, qy, qz, index, bank);
    p0.leafIndex = (int8_t)index;
    p0.bank = (int8_t)bank;
    return inew;
}

__device__ __forceinline__ const float2 *fpoly(const float (*a)[2]) { return reinterpret_cast<const float2 *>(a); }

__device__ uint32_t howfar_secjaws_y(const DevCtx &C, Part &p, float &t)
{
    const gegs_field *F = &C.fields[p.field];
    uint32_t inew = 0;
    float2 p0, p1 = make_float2(p.y, p.z), p2 = make_float2(p.x, p.z);
    float2 dir1 = make_float2(p.v, p.w), dir2 = make_float2(p.u, p.w);
    int inside_XZ, inside_YZ;
    float dis_xz = ray_intersect_polygon<false>(p1, dir1, fpoly(F->boundMaxY), 4, inside_XZ);
    float dis_yz = ray_intersect_polygon<false>(p2, dir2, fpoly(F->boundMaxY), 4, inside_YZ);
    float minBoundaryDist;
    if (dis_xz >= GX_INFI_DIST || dis_yz >= GX_INFI_DIST) return inew;
    if (dis_xz < dis_yz) minBoundaryDist = dis_xz; else minBoundaryDist = dis_yz;
    if (inside_XZ && inside_YZ) {
        if (point_in_polygon(p2, fpoly(F->jawsGeomY) + 2, 4)) {
            inew = 1;
            dis_xz = ray_intersect_polygon<false>(p2, dir2, fpoly(F->jawsGeomY), 4, inside_YZ);
            dis_yz = ray_intersect_polygon<false>(p2, dir2, fpoly(F->jawsGeomY) + 4, 4, inside_YZ);
            if (dis_xz < GX_INFI_DIST) {
                if (t > dis_xz) { inew = 2; t = dis_xz + GX_EPSTEP; }
            } else if (dis_yz < GX_INFI_DIST) {
                if (t > dis_yz) { inew = 2; t = dis_yz + GX_EPSTEP; }
            } else {
                if (t > minBoundaryDist) { t = minBoundaryDist + GX_EPSTEP; p.module = (uint8_t)C.module_order[GEGS_M_SECJAWY]; }
            }
        } else {
            inew = 2;
            dis_yz = ray_intersect_polygon<false>(p2, dir2, fpoly(F->jawsGeomY) + 2, 4, inside_YZ);
            if (dis_yz < GX_INFI_DIST) {
                if (t > dis_yz) { inew = 1; t = dis_yz + GX_EPSTEP; }
            } else {
                if (t > minBoundaryDist) { inew = 0; t = minBoundaryDist + GX_EPSTEP; }
            }
        }
    } else {
        inew = 1;
        if (t > minBoundaryDist) {
            t = minBoundaryDist + GX_EPSTEP;
            p0.x = p.y + t * p.v;
            p0.y = p.x + t * p.u;
            if (!point_in_polygon(p0, fpoly(F->boundMinY), 4)) inew = 0;
            else {
                p0.x = p0.y;
                p0.y = p.z + t * p.w;
                if (point_in_polygon(p0, fpoly(F->jawsGeomY) + 2, 4)) inew = 1;
                else inew = 2;
            }
        }
    }
    return inew;
}

__device__ uint32_t howfar_secjaws_x(const DevCtx &C, Part &p, float &t)
{
    const gegs_field *F = &C.fields[p.field];
    uint32_t inew = 0;
    float2 p0, p1 = make_float2(p.y, p.z), p2 = make_float2(p.x, p.z);
    float2 dir1 = make_float2(p.v, p.w), dir2 = make_float2(p.u, p.w);
    int inside_XZ, inside_YZ;
    float dis_xz = ray_intersect_polygon<false>(p1, dir1, fpoly(F->boundMaxX), 4, inside_XZ);
    float dis_yz = ray_intersect_polygon<false>(p2, dir2, fpoly(F->boundMaxX), 4, inside_YZ);
    float minBoundaryDist;
    if (dis_xz >= GX_INFI_DIST || dis_yz >= GX_INFI_DIST) return inew;
    if (dis_xz < dis_yz) minBoundaryDist = dis_xz; else minBoundaryDist = dis_yz;
    if (inside_XZ && inside_YZ) {
        if (point_in_polygon(p1, fpoly(F->jawsGeomX) + 2, 4)) {
            inew = 1;
            dis_xz = ray_intersect_polygon<false>(p1, dir1, fpoly(F->jawsGeomX), 4, inside_XZ);
            dis_yz = ray_intersect_polygon<false>(p1, dir1, fpoly(F->jawsGeomX) + 4, 4, inside_XZ);
            if (dis_xz < GX_INFI_DIST) {
                if (t > dis_xz) { inew = 2; t = dis_xz + GX_EPSTEP; }
            } else if (dis_yz < GX_INFI_DIST) {
                if (t > dis_yz) { inew = 2; t = dis_yz + GX_EPSTEP; }
            } else {
                if (t > minBoundaryDist) { t = minBoundaryDist + GX_EPSTEP; p.module = (uint8_t)C.module_order[GEGS_M_SECJAWX]; }
            }
        } else {
            inew = 2;
            dis_xz = ray_intersect_polygon<false>(p1, dir1, fpoly(F->jawsGeomX) + 2, 4, inside_XZ);
            if (dis_xz < GX_INFI_DIST) {
                if (t > dis_xz) { inew = 1; t = dis_yz + GX_EPSTEP; }
            } else {
                if (t > minBoundaryDist) { inew = 0; t = minBoundaryDist + GX_EPSTEP; }
            }
        }
    } else {
        inew = 1;
        if (t > minBoundaryDist) {
            t = minBoundaryDist + GX_EPSTEP;
            p0.x = p.y + t * p.v;
            p0.y = p.x + t * p.u;
            if (!point_in_polygon(p0, fpoly(F->boundMinX), 4)) inew = 0;
            else {
                p0.y = p.z + t * p.w;
                if (point_in_polygon(p0, fpoly(F->jawsGeomX) + 2, 4)) inew = 1;
                else inew = 2;
            }
        }
    }
    return inew;
}

// ---- hownear -----------------------------------------------------------------
__device__ __forceinline__ float dist2p(float2 v, float2 w) { return (v.x - w.x) * (v.x - w.x) + (v.y - w.y) * (v.y - w.y); }
__device__ __forceinline__ float distp(float2 v, float2 w) { return sqrtf((v.x - w.x) * (v.x - w.x) + (v.y - w.y) * (v.y - w.y)); }

// Squared distance whose sqrtf is point_dist_to_segment(p, v, w), term for term.
__device__ __forceinline__ float point_dist2_to_segment(float2 p, float2 v, float2 w)
{
    float l2 = dist2p(v, w);
    if (l2 == 0) return dist2p(p, v);
    float tn = (p.x - v.x) * (w.x - v.x) + (p.y - v.y) * (w.y - v.y);
    // t = fl(tn / l2) with l2 > 0: certainly negative (and not rounded to zero)
    // below -l2 * 1e-30, certainly above 1 beyond l2 * (1 + 2^-20); only the
    // projection case needs the quotient itself
    if (tn < -l2 * 1e-30f) return dist2p(p, v);
    if (tn > l2 * 1.00000095367431640625f) return dist2p(p, w);
    float t = tn / l2;
    if (t < 0) return dist2p(p, v);
    if (t > 1) return dist2p(p, w);
    float2 a = make_float2(v.x + t * (w.x - v.x), v.y + t * (w.y - v.y));
    return dist2p(p, a);
}

// Minimum edge distance of the polygon, capped at 1e9 (pointMinDistToPolygon,
// geom.cu:1175-1191). sqrtf is correctly rounded and monotonic, so the
// minimum of the edges' sqrtf equals sqrtf of the minimum squared distance:
// one square root per polygon instead of one per edge, same result.
template <bool LOCAL>
__device__ float point_min_dist_to_polygon(float2 p0, const float2 *poly, int n)
{
    float min2 = __int_as_float(0x7f800000);
    for (int i = 0; i < n; i++) {
        int j = i + 1;
        if (j >= n) j = 0;
        float2 a = LOCAL ? poly[i] : ld2(&poly[i]);
        float2 b = LOCAL ? poly[j] : ld2(&poly[j]);
        float d2 = point_dist2_to_segment(p0, a, b);
        if (d2 < min2) min2 = d2;
    }
    float d = sqrtf(min2);
    return d < 1e9f ? d : 1e9f;
}

__device__ void hownear_mlc(const DevCtx &C, Part &p, float &tperp)
{
    float2 p1 = make_float2(p.x, p.z), p2 = make_float2(p.y, p.z);
    int index;
    float tperp_xz = GX_INFI_DIST + 1, tperp_yz = GX_INFI_DIST + 1, bound;
    int inside_XZ, inside_YZ;
    if (p.leafIndex < -60) {
        inside_XZ = point_in_polygon_local(p1, C.boundaryXZ, 4);
        inside_YZ = point_in_polygon_local(p2, C.boundaryYZ, 4);
    } else { inside_XZ = 1; inside_YZ = 1; }
    // the distance to the MLC boundary is needed only outside the MLC (the
    // reference computes it first in every case; the result is the same)
    if (inside_XZ && inside_YZ) {
        if (p.leafIndex > GX_PASSMLC) index = p.leafIndex;
        else { index = index_of_leaf(C, p1); p.leafIndex = (int8_t)index; }
        // In a leaf column: the leaf's XZ cross section, then its YZ leaf-end
        // outline; in an air gap: the XZ cross sections of the two leaves on
        // either side. Two polygon distances either way, taken in one loop so
        // that lanes of both cases share it (each lane keeps the reference's
        // polygons and order).
        if (index >= 0 && p.bank < 0) p.bank = (int8_t)point_in_leaf(p2, endnode_of(C, p.field, index));
        if (index > -60) {
            const bool leaf = index >= 0;
            const float2 *yzp = nullptr;
            int nvyz = 17;
            if (leaf) {
                yzp = endnode_of(C, p.field, index);
                if (p.bank == 0) { yzp += 2; nvyz = 30; }
                else if (p.bank == 2) { yzp += 17; }
            }
            float dd[2];
            for (int k = 0; k < 2; k++) {
                const bool yz = leaf && k == 1;
                const float2 *poly = leaf ? (k == 0 ? C.crossXZ + index * 16 : yzp) : C.crossXZ + (-index - k) * 16;
                dd[k] = point_min_dist_to_polygon<false>(yz ? p2 : p1, poly, yz ? nvyz : 14);
            }
            if (leaf) { tperp_xz = dd[0]; tperp_yz = dd[1]; }
            else tperp_xz = dd[0] < dd[1] ? dd[0] : dd[1];
        }
        if (tperp_xz < tperp_yz) tperp = tperp_xz; else tperp = tperp_yz;
    } else {
        float bxz = point_min_dist_to_polygon<true>(p1, C.boundaryXZ, 4);
        float byz = point_min_dist_to_polygon<true>(p2, C.boundaryYZ, 4);
        if (bxz < byz) bound = bxz; else bound = byz;
        tperp = bound;
    }
}

__device__ void hownear_secjaws_y(const DevCtx &C, const Part &p, float &tperp)
{
    const gegs_field *F = &C.fields[p.field];
    float2 p1 = make_float2(p.y, p.z), p2 = make_float2(p.x, p.z);
    int inside_XZ = point_in_polygon(p1, fpoly(F->boundMaxY), 4);
    int inside_YZ = point_in_polygon(p2, fpoly(F->boundMaxY), 4);
    float bound_xz = point_min_dist_to_polygon<false>(p1, fpoly(F->boundMaxY), 4);
    float bound_yz = point_min_dist_to_polygon<false>(p2, fpoly(F->boundMaxY), 4);
    if (inside_XZ && inside_YZ) {
        float dist_yz = point_min_dist_to_polygon<false>(p2, fpoly(F->jawsGeomY) + 2, 4);
        if (point_in_polygon(p2, fpoly(F->jawsGeomY) + 2, 4)) {
            if (dist_yz < bound_xz) tperp = dist_yz; else tperp = bound_xz;
        } else {
            if (dist_yz > bound_yz) dist_yz = bound_yz;
            if (dist_yz < bound_xz) tperp = dist_yz; else tperp = bound_xz;
        }
    } else {
        if (bound_xz < bound_yz) tperp = bound_xz; else tperp = bound_yz;
    }
}

__device__ void hownear_secjaws_x(const DevCtx &C, const Part &p, float &tperp)
{
    const gegs_field *F = &C.fields[p.field];
    float2 p1 = make_float2(p.y, p.z), p2 = make_float2(p.x, p.z);
    int inside_XZ = point_in_polygon(p1, fpoly(F->boundMaxX), 4);
    int inside_YZ = point_in_polygon(p2, fpoly(F->boundMaxX), 4);
    float bound_xz = point_min_dist_to_polygon<false>(p1, fpoly(F->boundMaxX), 4);
    float bound_yz = point_min_dist_to_polygon<false>(p2, fpoly(F->boundMaxX), 4);
    if (inside_XZ && inside_YZ) {
        float dist_xz = point_min_dist_to_polygon<false>(p1, fpoly(F->jawsGeomX) + 2, 4);
        if (point_in_polygon(p1, fpoly(F->jawsGeomX) + 2, 4)) {
            if (dist_xz < bound_yz) tperp = dist_xz; else tperp = bound_yz;
        } else {
            if (dist_xz > bound_xz) dist_xz = bound_xz;
            if (dist_xz < bound_yz) tperp = dist_xz; else tperp = bound_yz;
        }
    } else {
        if (bound_xz < bound_yz) tperp = bound_xz; else tperp = bound_yz;
    }
}

// Lower bound on hownear_secjaws_y / _x: their result is a minimum over
// distances to some of three (point, polygon) pairs -- the bounding polygon
// seen from (y, z) and from (x, z), and the jaw opening seen from (x, z) for
// the Y jaws or from (y, z) for the X jaws -- and a distance to a polygon is
// at least the distance to the line of its nearest edge. 10 um covers the
// rounding of both sides at coordinates up to 100 cm (a few 1e-5 cm). Every
// lane evaluates the same twelve lines, so a warp whose steps are all shorter
// than the bound skips the exact polygon distances as a whole.
__device__ __forceinline__ float jaws_near_lower_bound(const DevCtx &C, const Part &p)
{
    const bool xjaw = p.module == GEGS_M_SECJAWX;
    const float4 *L = C.jaw_lines + ((size_t)p.field * 2 + (xjaw ? 1 : 0)) * 8;
    float m = __int_as_float(0x7f7fffff);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float4 l = __ldg(&L[k]);
        m = fminf(m, fabsf(l.x * p.y + l.y * p.z - l.z));
        m = fminf(m, fabsf(l.x * p.x + l.y * p.z - l.z));
    }
    const float qx = xjaw ? p.y : p.x;
#pragma unroll
    for (int k = 4; k < 8; k++) {
        const float4 l = __ldg(&L[k]);
        m = fminf(m, fabsf(l.x * qx + l.y * p.z - l.z));
    }
    return m - 1e-3f;
}

// dispatch on the particle's module (photon.cu:142-158, electron.cu:1491-1508)
__device__ __forceinline__ uint32_t howfar(const DevCtx &C, Part &p, float &t, bool &ok)
{
    ok = true;
    switch (p.module) {
    case GEGS_M_PHANTOM: return howfar_phantom(C, p, t);
    case GEGS_M_VARMLC: return howfar_mlc(C, p, t);
    case GEGS_M_SECJAWY: return howfar_secjaws_y(C, p, t);
    case GEGS_M_SECJAWX: return howfar_secjaws_x(C, p, t);
    default: ok = false; return 0;
    }
}

__device__ __forceinline__ void hownear(const DevCtx &C, Part &p, float &tperp, bool &ok)
{
    ok = true;
    switch (p.module) {
    case GEGS_M_PHANTOM: hownear_phantom(C, p, tperp); return;
    case GEGS_M_VARMLC: hownear_mlc(C, p, tperp); return;
    case GEGS_M_SECJAWY: hownear_secjaws_y(C, p, tperp); return;
    case GEGS_M_SECJAWX: hownear_secjaws_x(C, p, tperp); return;
    default: ok = false; tperp = 0; return;
    }
}

// Geometry classes: a consumer kernel compiled for one class contains only that
// class's geometry code -- the secondary jaws, the MLC, or the phantom voxels --
// which keeps the code a divergent warp runs small. Classes are numbered in beam
// order; a particle whose module is outside the class is handed to the other
// class's kernel between steps. GX_GEOM_ALL compiles every module (plain form).
#define GX_GEOM_ALL 0
#define GX_GEOM_JAWS 1
#define GX_GEOM_MLC 2
#define GX_GEOM_PHANTOM 3

// class of a module (unsupported modules fall in the jaws class, whose
// geometry dispatch reports them)
__device__ __forceinline__ int geom_class_of(uint8_t module)
{
    if (module == GEGS_M_PHANTOM) return GX_GEOM_PHANTOM;
    if (module == GEGS_M_VARMLC) return GX_GEOM_MLC;
    return GX_GEOM_JAWS;
}

template <int G>
__device__ __forceinline__ bool in_geom_class(const Part &p)
{
    return G == GX_GEOM_ALL || geom_class_of(p.module) == G;
}

template <int G>
__device__ __forceinline__ uint32_t howfar_g(const DevCtx &C, Part &p, float &t, bool &ok)
{
    if (G == GX_GEOM_ALL) return howfar(C, p, t, ok);
    ok = true;
    if (G == GX_GEOM_PHANTOM) {
        if (p.module == GEGS_M_PHANTOM) return howfar_phantom(C, p, t);
    } else if (G == GX_GEOM_MLC) {
        if (p.module == GEGS_M_VARMLC) return howfar_mlc(C, p, t);
    } else {
        if (p.module == GEGS_M_SECJAWY) return howfar_secjaws_y(C, p, t);
        if (p.module == GEGS_M_SECJAWX) return howfar_secjaws_x(C, p, t);
    }
    ok = false;
    return 0;
}

template <int G>
__device__ __forceinline__ void hownear_g(const DevCtx &C, Part &p, float &tperp, bool &ok)
{
    if (G == GX_GEOM_ALL) { hownear(C, p, tperp, ok); return; }
    ok = true;
    if (G == GX_GEOM_PHANTOM) {
        if (p.module == GEGS_M_PHANTOM) { hownear_phantom(C, p, tperp); return; }
    } else if (G == GX_GEOM_MLC) {
        if (p.module == GEGS_M_VARMLC) { hownear_mlc(C, p, tperp); return; }
    } else {
        if (p.module == GEGS_M_SECJAWY) { hownear_secjaws_y(C, p, tperp); return; }
        if (p.module == GEGS_M_SECJAWX) { hownear_secjaws_x(C, p, tperp); return; }
    }
    ok = false;
    tperp = 0;
}
