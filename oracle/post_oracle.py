"""Oracle (test infrastructure) for the dose interpolation: a restatement of
the reference's interp_dose (output.c:221-316) pass by pass -- z, then y, then
x -- in float32 on small grids. The reference keeps the intermediate passes in
place in the output buffer; here each pass has its own array, which gives the
values the reference computes when the output grid is at least as large as the
phantom in x and y (its in-place layout needs that)."""
import numpy as np


def interp_dose(dose, x_bounds, y_bounds, z_bounds, start, sizes, dims):
    f = np.float32
    nx, ny, nz = len(x_bounds) - 1, len(y_bounds) - 1, len(z_bounds) - 1
    d = np.asarray(dose, np.float32).reshape(nz, ny, nx)
    c = [((np.asarray(b, np.float32)[:-1] + np.asarray(b, np.float32)[1:]) / f(2)).astype(np.float32)
         for b in (x_bounds, y_bounds, z_bounds)]
    xc, yc, zc = c
    mx, my, mz = dims
    sx, sy, sz = (f(v) for v in sizes)
    x0, y0, z0 = (f(v) for v in start)
    A = np.zeros((mz, ny, nx), np.float32)                       # z pass (output.c:238-260)
    for iz in range(mz):
        z = f(z0 + sz * f(iz))
        if z <= zc[0] or z >= zc[nz - 1]:
            continue
        for k in range(nz - 1):
            if zc[k] < z <= zc[k + 1]:
                A[iz] = d[k] + (z - zc[k]) * (d[k + 1] - d[k]) / (zc[k + 1] - zc[k])
                break
    B = np.zeros((mz, my, nx), np.float32)                       # y pass (output.c:262-284)
    for iy in range(my):
        y = f(y0 + sy * f(iy))
        if y <= yc[0] or y >= yc[ny - 1]:
            continue
        for j in range(ny - 1):
            if yc[j] < y <= yc[j + 1]:
                B[:, iy] = A[:, j] + (y - yc[j]) * (A[:, j + 1] - A[:, j]) / (yc[j + 1] - yc[j])
                break
    out = np.zeros((mz, my, mx), np.float32)                     # x pass (output.c:286-303)
    for ix in range(mx):
        x = f(x0 + sx * f(ix))
        if x <= xc[0] or x >= xc[nx - 1]:
            continue
        for i in range(nx - 1):
            if xc[i] < x <= xc[i + 1]:
                out[:, :, ix] = B[:, :, i] + (x - xc[i]) * (B[:, :, i + 1] - B[:, :, i]) / (xc[i + 1] - xc[i])
                break
    return out
