// Dose post-processing and phantom preparation on the GPU:
//   gegs_interp_dose   separable linear interpolation of the dose grid between
//                      voxel centres (interp_dose, output.c:221-316);
//   gegs_gamma3d       3-D global gamma index (dose difference + distance to
//                      agreement) of an evaluated dose against a reference dose;
//   gegs_ct_ramp       HU -> (medium, density) through a piecewise-linear ramp
//                      (CTToMedium's 4-material ramp, ctcreate.c:913-970,1057-1104).
// Host buffers in and out; device memory is allocated per call.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>
#include "../../include/gegs_post.h"

namespace {

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

// ---- interpolation -------------------------------------------------------
// Voxel centres are (b[i] + b[i+1]) / 2 in float, as the reference computes
// them. A coordinate at or beyond the first or last centre gives 0. Per output
// point the z, then y, then x interpolation is done with the reference's
// operations in the reference's order.
__device__ __forceinline__ int bracket(const float *c, int n, float v)
{
    // first k with c[k] < v <= c[k+1]; the caller has checked c[0] < v < c[n-1]
    int lo = 0, hi = n - 2;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (c[mid] < v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_interp(const float *__restrict__ d, int nx, int ny, int nz, const float *xc, const float *yc,
                         const float *zc, float x0, float y0, float z0, float sx, float sy, float sz, int mx, int my,
                         int mz, float *out)
{
    long long n = (long long)mx * my * mz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(t % mx), iy = (int)((t / mx) % my), iz = (int)(t / ((long long)mx * my));
        float x = x0 + sx * ix, y = y0 + sy * iy, z = z0 + sz * iz;
        float v = 0.0f;
        if (z > zc[0] && z < zc[nz - 1] && y > yc[0] && y < yc[ny - 1] && x > xc[0] && x < xc[nx - 1]) {
            int k = bracket(zc, nz, z), j = bracket(yc, ny, y), i = bracket(xc, nx, x);
            long long pxy = (long long)nx * ny;
            float dz[2][2];
            for (int b = 0; b < 2; b++)
                for (int a = 0; a < 2; a++) {
                    long long c = (i + a) + (long long)nx * (j + b) + pxy * k;
                    float d0 = d[c], d1 = d[c + pxy];
                    dz[b][a] = d0 + (z - zc[k]) * (d1 - d0) / (zc[k + 1] - zc[k]);
                }
            float dy0 = dz[0][0] + (y - yc[j]) * (dz[1][0] - dz[0][0]) / (yc[j + 1] - yc[j]);
            float dy1 = dz[0][1] + (y - yc[j]) * (dz[1][1] - dz[0][1]) / (yc[j + 1] - yc[j]);
            v = dy0 + (x - xc[i]) * (dy1 - dy0) / (xc[i + 1] - xc[i]);
        }
        out[t] = v;
    }
}

// ---- gamma ---------------------------------------------------------------
// For every reference voxel with dose >= cutoff, the minimum over evaluated
// voxels within the search list of  d2 / dta^2 + (E - R)^2 / dd^2, where the
// list holds the integer offsets with their squared distance d2, sorted by d2;
// the scan stops when d2 / dta^2 alone reaches the best value found.
__global__ void k_gamma(const float *__restrict__ ref, const float *__restrict__ ev, int nx, int ny, int nz,
                        const int4 *off, const float *off_d2, int noff, float inv_dta2, float inv_dd2, float cutoff,
                        float *gamma, unsigned long long *counts)
{
    long long n = (long long)nx * ny * nz;
    unsigned long long ne = 0, np = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        float r = ref[t];
        if (!(r >= cutoff)) { gamma[t] = -1.0f; continue; }
        int ix = (int)(t % nx), iy = (int)((t / nx) % ny), iz = (int)(t / ((long long)nx * ny));
        float best = __int_as_float(0x7f800000);
        for (int k = 0; k < noff; k++) {
            float g_r = off_d2[k] * inv_dta2;
            if (g_r >= best) break;
            int4 o = off[k];
            int x = ix + o.x, y = iy + o.y, z = iz + o.z;
            if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
            float e = ev[x + (long long)nx * y + (long long)nx * ny * z];
            float dd = e - r;
            float g = g_r + dd * dd * inv_dd2;
            if (g < best) best = g;
        }
        float gv = sqrtf(best);
        gamma[t] = gv;
        ne++;
        if (gv <= 1.0f) np++;
    }
    for (int s = 16; s > 0; s >>= 1) {
        ne += __shfl_down_sync(0xffffffffu, ne, s);
        np += __shfl_down_sync(0xffffffffu, np, s);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counts[0], ne);
        atomicAdd(&counts[1], np);
    }
}

// ---- CT ramp --------------------------------------------------------------
__global__ void k_ct_ramp(const int16_t *__restrict__ hu, long long n, const gegs_ct_ramp_segment *seg, int nseg,
                          double hu_lower, uint16_t *med, float *dens)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double h = (double)hu[t];
        uint16_t m = 0xFFFFu;
        double d = 0.0;
        if (h > seg[nseg - 1].hu_upper) {
            m = (uint16_t)seg[nseg - 1].medium;
            d = seg[nseg - 1].density_upper;
        } else if (!(h < hu_lower)) {
            double lower = hu_lower;
            for (int s = 0; s < nseg; s++) {
                if (h <= seg[s].hu_upper) {
                    m = (uint16_t)seg[s].medium;
                    d = seg[s].density_lower + (h - lower) * (seg[s].density_upper - seg[s].density_lower)
                        / (seg[s].hu_upper - lower);
                    break;
                }
                lower = seg[s].hu_upper;
            }
        }
        med[t] = m;
        dens[t] = (float)d;
    }
}

#define PK(call)                                                                   \
    do {                                                                           \
        cudaError_t _c = (call);                                                   \
        if (_c != cudaSuccess) {                                                   \
            fprintf(stderr, "gegs post-processing: %s: %s\n", #call, cudaGetErrorString(_c)); \
            return _c == cudaErrorMemoryAllocation ? 5 : 2;                        \
        }                                                                          \
    } while (0)

template <typename T>
int dev_copy(DevBuf &b, const T *h, size_t n)
{
    PK(cudaMalloc(&b.p, n * sizeof(T) + 16));
    if (h) PK(cudaMemcpy(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

int grid_for(long long n)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long g = (n + 255) / 256;
    long long cap = (long long)nsm * 8;
    return (int)(g < cap ? (g > 0 ? g : 1) : cap);
}

}  // namespace

extern "C" int gegs_interp_dose(int device, const float *dose, int nx, int ny, int nz, const float *x_bounds,
                                const float *y_bounds, const float *z_bounds, float x0, float y0, float z0, float sx,
                                float sy, float sz, int mx, int my, int mz, float *out)
{
    if (!dose || !out || !x_bounds || !y_bounds || !z_bounds || nx < 2 || ny < 2 || nz < 2 || mx <= 0 || my <= 0 || mz <= 0)
        return 1;
    PK(cudaSetDevice(device));
    std::vector<float> c[3];
    const float *b[3] = {x_bounds, y_bounds, z_bounds};
    int nn[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) {
        c[a].resize(nn[a]);
        for (int i = 0; i < nn[a]; i++) c[a][i] = (b[a][i] + b[a][i + 1]) / 2;
    }
    long long nin = (long long)nx * ny * nz, nout = (long long)mx * my * mz;
    DevBuf dd, dx, dy, dz, dout;
    int st;
    if ((st = dev_copy(dd, dose, (size_t)nin)) || (st = dev_copy(dx, c[0].data(), nx)) ||
        (st = dev_copy(dy, c[1].data(), ny)) || (st = dev_copy(dz, c[2].data(), nz)) ||
        (st = dev_copy<float>(dout, nullptr, (size_t)nout)))
        return st;
    k_interp<<<grid_for(nout), 256>>>((const float *)dd.p, nx, ny, nz, (const float *)dx.p, (const float *)dy.p,
                                      (const float *)dz.p, x0, y0, z0, sx, sy, sz, mx, my, mz, (float *)dout.p);
    PK(cudaGetLastError());
    PK(cudaMemcpy(out, dout.p, (size_t)nout * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int gegs_gamma3d(int device, const float *ref, const float *eval, int nx, int ny, int nz, float dx, float dy,
                            float dz, float dta, float dd_abs, float cutoff_abs, float search_dta, float *gamma,
                            uint64_t *n_evaluated, uint64_t *n_passed)
{
    if (!ref || !eval || !gamma || nx <= 0 || ny <= 0 || nz <= 0 || !(dta > 0) || !(dd_abs > 0) || !(search_dta > 0))
        return 1;
    PK(cudaSetDevice(device));
    // offsets within search_dta * dta, sorted by squared distance (float arithmetic as the kernel's)
    float rmax = search_dta * dta;
    int rx = (int)(rmax / dx), ry = (int)(rmax / dy), rz = (int)(rmax / dz);
    std::vector<std::pair<float, int4>> offs;
    for (int k = -rz; k <= rz; k++)
        for (int j = -ry; j <= ry; j++)
            for (int i = -rx; i <= rx; i++) {
                float px = dx * (float)i, py = dy * (float)j, pz = dz * (float)k;
                float d2 = px * px + py * py + pz * pz;
                if (d2 <= rmax * rmax) offs.push_back({d2, make_int4(i, j, k, 0)});
            }
    std::stable_sort(offs.begin(), offs.end(), [](const std::pair<float, int4> &a, const std::pair<float, int4> &b) {
        return a.first < b.first;
    });
    std::vector<int4> o4(offs.size());
    std::vector<float> o2(offs.size());
    for (size_t k = 0; k < offs.size(); k++) { o4[k] = offs[k].second; o2[k] = offs[k].first; }
    long long n = (long long)nx * ny * nz;
    DevBuf dr, de, dg, doff, dod2, dcnt;
    int st;
    if ((st = dev_copy(dr, ref, (size_t)n)) || (st = dev_copy(de, eval, (size_t)n)) ||
        (st = dev_copy<float>(dg, nullptr, (size_t)n)) || (st = dev_copy(doff, o4.data(), o4.size())) ||
        (st = dev_copy(dod2, o2.data(), o2.size())) || (st = dev_copy<unsigned long long>(dcnt, nullptr, 2)))
        return st;
    PK(cudaMemset(dcnt.p, 0, 2 * sizeof(unsigned long long)));
    k_gamma<<<grid_for(n), 256>>>((const float *)dr.p, (const float *)de.p, nx, ny, nz, (const int4 *)doff.p,
                                  (const float *)dod2.p, (int)o4.size(), 1.0f / (dta * dta),
                                  1.0f / (dd_abs * dd_abs), cutoff_abs, (float *)dg.p, (unsigned long long *)dcnt.p);
    PK(cudaGetLastError());
    unsigned long long cnt[2];
    PK(cudaMemcpy(cnt, dcnt.p, sizeof cnt, cudaMemcpyDeviceToHost));
    PK(cudaMemcpy(gamma, dg.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    if (n_evaluated) *n_evaluated = cnt[0];
    if (n_passed) *n_passed = cnt[1];
    return 0;
}

extern "C" int gegs_ct_ramp(int device, const int16_t *hu, uint64_t n, const gegs_ct_ramp_segment *segments,
                            int nseg, double hu_lower, uint16_t *medium, float *density)
{
    if (!hu || !segments || nseg <= 0 || !medium || !density) return 1;
    PK(cudaSetDevice(device));
    DevBuf dh, ds, dm, dd;
    int st;
    if ((st = dev_copy(dh, hu, (size_t)n)) || (st = dev_copy(ds, segments, (size_t)nseg)) ||
        (st = dev_copy<uint16_t>(dm, nullptr, (size_t)n)) || (st = dev_copy<float>(dd, nullptr, (size_t)n)))
        return st;
    k_ct_ramp<<<grid_for((long long)n), 256>>>((const int16_t *)dh.p, (long long)n, (const gegs_ct_ramp_segment *)ds.p,
                                               nseg, hu_lower, (uint16_t *)dm.p, (float *)dd.p);
    PK(cudaGetLastError());
    PK(cudaMemcpy(medium, dm.p, (size_t)n * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    PK(cudaMemcpy(density, dd.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}
