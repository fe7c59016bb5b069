/* A second, independent statement of the reference's comparison of a dose
 * grid with detector-array data (output_RelDos_II, output.c:596-778), in
 * plain C with C's own float semantics, for checking the package's
 * postprocess.relative_dose. Test infrastructure: compiled and run by
 * tests/test_reldose.py.
 *
 *   reldose DOSE BOUNDS NX NY NZ X0 Y0 Z0 SX SY SZ MX MY MZ MEAS NORM ARRAY LEN DOS IX IY IZ OUT
 *
 * DOSE is the raw float32 dose grid (x fastest), BOUNDS the nx+1, ny+1, nz+1
 * voxel boundaries as raw float32. Real arguments are read with strtof (hex
 * floats keep them exact). MEAS is the measured data file, "-" for none.
 * NORM 1 normalises to the maxima, 2 to the isocentre point (IX IY IZ), any
 * other value compares measured data * 100 directly. ARRAY 1 compares point
 * by point (PTW729); otherwise neighbours along x and z may rescue a point
 * (PTW1000). LEN (cm) and DOS (fraction) are the gamma criteria. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

static float *read_floats(const char *path, size_t n)
{
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    float *v = malloc(n * sizeof(float));
    size_t got = fread(v, sizeof(float), n, f);
    fclose(f);
    if (got != n) { free(v); return NULL; }
    return v;
}

/* Voxel centres, (b[i] + b[i+1]) / 2 in float, as the reference keeps them
 * after reading the phantom (init.cu:1308-1312). */
static void centres(const float *b, int n, float *c)
{
    for (int i = 0; i < n; i++) c[i] = (b[i] + b[i + 1]) / 2;
}

/* The index of the grid point's voxel, truncating (p - c0) / (c1 - c0) + 0.1
 * (the 0.1 is a double literal, so the sum is a double). */
static int nearest(float p, const float *c)
{
    float r = (p - c[0]) / (c[1] - c[0]);
    return (int)(r + 0.1);
}

/* The gamma-like test against a neighbour's calculated dose: the dose
 * difference in units of DOS, squared in float, then the distance term in
 * double (0.25 * 0.25 / len / len is a double expression). */
static int neighbour_agrees(float calc, float meas, float dos, float len)
{
    float g = fabsf(calc - meas) / meas / dos;
    g = g * g;
    g = (float)sqrt(g + 0.25 * 0.25 / len / len);
    return g <= 1;
}

int main(int argc, char **argv)
{
    if (argc != 24) { fprintf(stderr, "usage: see the header of reldose.c\n"); return 2; }
    const int nx = atoi(argv[3]), ny = atoi(argv[4]), nz = atoi(argv[5]);
    const float x0 = strtof(argv[6], NULL), y0 = strtof(argv[7], NULL), z0 = strtof(argv[8], NULL);
    const float sx = strtof(argv[9], NULL), sy = strtof(argv[10], NULL), sz = strtof(argv[11], NULL);
    const int mx = atoi(argv[12]), my = atoi(argv[13]), mz = atoi(argv[14]);
    const char *meas_path = argv[15];
    const int norm = atoi(argv[16]), array = atoi(argv[17]);
    const float len = strtof(argv[18], NULL), dos = strtof(argv[19], NULL);
    const float ix = strtof(argv[20], NULL), iy = strtof(argv[21], NULL), iz = strtof(argv[22], NULL);
    const size_t nvox = (size_t)nx * ny * nz, npt = (size_t)mx * my * mz;

    float *dose = read_floats(argv[1], nvox);
    float *bounds = read_floats(argv[2], (size_t)nx + ny + nz + 3);
    if (!dose || !bounds) { fprintf(stderr, "cannot read the dose grid or the bounds\n"); return 1; }
    float *cx = malloc(nx * sizeof(float)), *cy = malloc(ny * sizeof(float)), *cz = malloc(nz * sizeof(float));
    centres(bounds, nx, cx);
    centres(bounds + nx + 1, ny, cy);
    centres(bounds + nx + ny + 2, nz, cz);

    /* calculated dose at each grid point */
    float *calc = malloc(npt * sizeof(float));
    for (int k = 0; k < mz; k++)
        for (int j = 0; j < my; j++)
            for (int i = 0; i < mx; i++) {
                const int vx = nearest(x0 + sx * i, cx), vy = nearest(y0 + sy * j, cy), vz = nearest(z0 + sz * k, cz);
                if (vx < 0 || vx >= nx || vy < 0 || vy >= ny || vz < 0 || vz >= nz) {
                    fprintf(stderr, "grid point outside the phantom\n");
                    return 1;
                }
                calc[((size_t)k * my + j) * mx + i] = dose[((size_t)vz * ny + vy) * nx + vx];
            }

    FILE *out = fopen(argv[23], "w");
    if (!out) return 1;
    FILE *mf = meas_path[0] == '-' ? NULL : fopen(meas_path, "r");
    if (!mf) {                       /* no measured data: the sampled doses alone */
        for (size_t i = 0; i < npt; i++) fprintf(out, "%f\n", calc[i]);
        fclose(out);
        return 0;
    }

    /* measured data: the first number of each line, rounded once to float */
    float *meas = malloc(npt * sizeof(float));
    char line[4096];
    size_t got = 0;
    while (got < npt && fgets(line, sizeof line, mf)) {
        char *end;
        float v = strtof(line, &end);
        if (end != line) meas[got++] = v;
    }
    fclose(mf);
    if (got < npt) { fprintf(stderr, "measured data: %zu values, %zu expected\n", got, npt); return 1; }

    float top_meas = 0.0f, top_calc = 0.0f;   /* running maxima from 0, as the reference keeps them */
    for (size_t i = 0; i < npt; i++) {
        if (norm != 1 && norm != 2) meas[i] = meas[i] * 100.0f;
        if (meas[i] > top_meas) top_meas = meas[i];
        if (calc[i] > top_calc) top_calc = calc[i];
    }
    if (norm == 1) {
        for (size_t i = 0; i < npt; i++) { meas[i] = meas[i] / top_meas; calc[i] = calc[i] / top_calc; }
        top_meas = 1.0f;
    } else if (norm == 2) {
        size_t c = 0;
        if (sx != 0) c += (size_t)(int)((ix - x0) / sx + 0.1);
        if (sy != 0) c += (size_t)(int)((iy - y0) / sy + 0.1) * mx;
        if (sz != 0) c += (size_t)(int)((iz - z0) / sz + 0.1) * mx * my;
        const float mc = meas[c], cc = calc[c];
        for (size_t i = 0; i < npt; i++) { meas[i] = meas[i] / mc; calc[i] = calc[i] / cc; }
        top_meas = top_meas / mc;
    }
    const float threshold = top_meas * 0.1f;

    unsigned compared = 0, passed = 0;
    for (size_t i = 0; i < npt; i++) {
        int verdict = 0;
        const float m = meas[i];
        if (m > threshold) {
            compared++;
            const int ok = fabsf(calc[i] - m) / m <= dos;
            if (array == 1) {
                verdict = ok ? 1 : -1;
            } else {
                const int row = (int)(i / mx), col = (int)(i - (size_t)row * mx);
                verdict = ok;
                /* the reference asks the x neighbours and the next z neighbour
                 * only while nothing has passed yet, the previous z neighbour
                 * always (output.c:729-756) */
                if (col > 0 && verdict <= 0) verdict += neighbour_agrees(calc[i - 1], m, dos, len);
                if (col + 1 < mx && verdict <= 0) verdict += neighbour_agrees(calc[i + 1], m, dos, len);
                if (row > 0) verdict += neighbour_agrees(calc[i - mx], m, dos, len);
                if (row + 1 < mz && verdict <= 0) verdict += neighbour_agrees(calc[i + mx], m, dos, len);
                if (verdict <= 0) verdict = -1;
            }
            if (verdict > 0) passed++;
        }
        fprintf(out, "%f\t %f\t %d\n", m, calc[i], verdict);
    }
    const float share = (float)passed / compared;
    fprintf(out, "Totally %u points compared, %u passed, percentage = %.0f %%\n", compared, passed, share * 100);
    fclose(out);
    return 0;
}
