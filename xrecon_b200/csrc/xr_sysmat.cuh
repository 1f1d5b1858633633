// Sparse export of the projection matrix A (the reference's
// system_matrix2d/3d, src/cpu/system_matrix2d.cpp:369-396 and
// src/cpu/system_matrix3d.cpp:39-62 over the visitor of
// src/cpu/forward3d.cpp:611-660): one thread per detector cell walks the
// lines of its view and emits every (cell, voxel) weight of the projection,
// in two passes: COUNT writes the number of nonzero weights of each cell,
// FILL writes them at the offsets of an exclusive scan of those counts.
//
//   row = (view * Nv + det_row) * Nu + physical column   (2D: view * Nu + column)
//   col = (iz * H + iy) * W + ix                          (2D: iy * W + ix)
//   value = s_A(k, r) * lf(L) * overlap_xy * overlap_z   (FP64, stored as FP32)
//
// Cells are numbered (view, det_row, traversal column k); the weights are the
// ones the cell gathers accumulate, so A_sparse x equals the projection of x.
// Zero weights are skipped, as in the reference.
#pragma once

#include "xr_kernels.cuh"

namespace xr {

template <bool FILL, bool DIM3>
__global__ void __launch_bounds__(128)
sysmat_kernel(const Geom g, const ViewTables vt, const int nview, long long* __restrict__ counts,
              const long long* __restrict__ offsets, long long* __restrict__ rows, long long* __restrict__ cols,
              float* __restrict__ vals, const double z0dz, const double zd0, const double dvv) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int Nu = g.Nu, Nv = DIM3 ? g.Nv : 1;
    if (c >= (long long)nview * Nv * Nu) return;
    const int k = (int)(c % Nu);
    const int r = (int)((c / Nu) % Nv);
    const int v = (int)(c / ((long long)Nu * Nv));
    const ViewHdr h = vt.hdr[v];
    const size_t ob = (size_t)v * (Nu + 1) + k;
    const double bA0 = vt.bA[ob], bB0 = vt.bB[ob], bA1 = vt.bA[ob + 1], bB1 = vt.bB[ob + 1];
    const size_t oc = (size_t)v * Nu + k;
    // the cell scale, as the projection kernels apply it (FP32)
    float sA = vt.colE[oc];
    double Qk = 0.0;
    if (DIM3) {
        const float zc = (float)(zd0 + (r + 0.5) * dvv) * vt.colM[oc];
        sA *= sqrtf(vt.colF[oc] + zc * zc);
        Qk = vt.colQ[oc];
    }
    const int col = h.keep ? k : Nu - 1 - k;
    const long long row = ((long long)v * Nv + r) * Nu + col;
    long long n = 0;
    long long pos = FILL ? offsets[c] : 0;
    for (int L = 0; L < h.nlines; ++L) {
        const double pk = fma(bB0, (double)L, bA0);
        const double pk1 = fma(bB1, (double)L, bA1);
        const int pa = max((int)floor(pk), 0);
        const int pb = min((int)ceil(pk1) - 1, h.npix - 1);
        if (pa > pb) continue;
        const double q = fma(h.q1, (double)L, h.q0);
        double lf, tl = 0.0, th = 1.0;
        int ja = 0, jb = 0;
        if (DIM3) {
            lf = h.dpix * g.dz / (q * q);
            const double gq = Qk * q;
            tl = fma(gq, zd0 + r * dvv, -z0dz);
            th = fma(gq, zd0 + (r + 1) * dvv, -z0dz);
            if (th < tl) { const double t = tl; tl = th; th = t; }
            ja = max((int)floor(tl), 0);
            jb = min((int)floor(th), g.D - 1);
            if (ja > jb) continue;
        } else {
            lf = h.dpix / q;
        }
        for (int p = pa; p <= pb; ++p) {
            const double wx = fmin((double)p + 1.0, pk1) - fmax((double)p, pk);
            if (!(wx > 0.0)) continue;
            int ix, iy;
            if (h.use_x) { ix = p; iy = L; } else { ix = L; iy = g.H - 1 - p; }
            for (int j = ja; j <= jb; ++j) {
                const double wz = DIM3 ? fmin((double)j + 1.0, th) - fmax((double)j, tl) : 1.0;
                if (!(wz > 0.0)) continue;
                const float val = (float)((double)sA * lf * wx * wz);
                if (val == 0.0f) continue;
                if (FILL) {
                    rows[pos] = row;
                    cols[pos] = ((long long)j * g.H + iy) * g.W + ix;
                    vals[pos] = val;
                    ++pos;
                } else {
                    ++n;
                }
            }
        }
    }
    if (!FILL) counts[c] = n;
}

}  // namespace xr
