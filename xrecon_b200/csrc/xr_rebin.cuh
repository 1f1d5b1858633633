// Fan/cone -> parallel rebinning along the detector columns (the reference's
// fan_to_parallel_rebin, xrecon/utils/rebin.py:10-95).  The sampling grid
// (one normalized (x: column, y: view) pair per output view and parallel bin,
// the reference's `grid`) is computed by the caller; the kernels sample each
// detector row's [view][column] plane bilinearly with zero padding outside,
// with torch.nn.functional.grid_sample's align_corners=True convention:
//   ix = (x + 1) / 2 * (Nu - 1),  iy = (y + 1) / 2 * (V - 1),
// and corner weights (ix0 + 1 - ix)(iy0 + 1 - iy), (ix - ix0)(iy0 + 1 - iy),
// (ix0 + 1 - ix)(iy - iy0), (ix - ix0)(iy - iy0) for the corners
// (iy0, ix0), (iy0, ix0 + 1), (iy0 + 1, ix0), (iy0 + 1, ix0 + 1).
#pragma once

#include "xr_kernels.cuh"

namespace xr {

struct RebinGrid {
    const float* grid;  // [Vout][Nt][2]
    int V, Nv, Nu, Vout, Nt;
};

// Sample of the fan sinogram `src` (one batch element, [V][Nv][Nu]) at
// detector row `row` for output view vo and parallel bin t.
template <typename TI>
__device__ __forceinline__ float rebin_sample(const TI* __restrict__ src, const RebinGrid& r, int row, int vo, int t) {
    const float2 gxy = *reinterpret_cast<const float2*>(r.grid + 2 * ((size_t)vo * r.Nt + t));
    const float ix = (gxy.x + 1.0f) / 2.0f * (float)(r.Nu - 1);
    const float iy = (gxy.y + 1.0f) / 2.0f * (float)(r.V - 1);
    const float fx = floorf(ix), fy = floorf(iy);
    const int x0 = (int)fx, y0 = (int)fy;
    const float ax = fx + 1.0f - ix, bx = ix - fx, ay = fy + 1.0f - iy, by = iy - fy;
    float v = 0.0f;
    const bool x0in = x0 >= 0 && x0 < r.Nu, x1in = x0 + 1 >= 0 && x0 + 1 < r.Nu;
    if (y0 >= 0 && y0 < r.V) {
        const TI* p = src + ((size_t)y0 * r.Nv + row) * r.Nu;
        if (x0in) v += ld(p + x0) * (ax * ay);
        if (x1in) v += ld(p + x0 + 1) * (bx * ay);
    }
    if (y0 + 1 >= 0 && y0 + 1 < r.V) {
        const TI* p = src + ((size_t)(y0 + 1) * r.Nv + row) * r.Nu;
        if (x0in) v += ld(p + x0) * (ax * by);
        if (x1in) v += ld(p + x0 + 1) * (bx * by);
    }
    return v;
}

// Plain rebinning: one thread per output sample; grid (bins / 256, detector
// rows, output views x batch elements from z0), output [nbatch][Vout][Nv][Nt].
template <typename TI>
__global__ void __launch_bounds__(256)
rebin_kernel(const TI* __restrict__ in, float* __restrict__ out, const RebinGrid r, const int z0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= r.Nt) return;
    const int row = blockIdx.y;
    const int zb = z0 + blockIdx.z;             // b * Vout + vo
    const int vo = zb % r.Vout, b = zb / r.Vout;
    out[((size_t)zb * r.Nv + row) * r.Nt + t] = rebin_sample(in + (size_t)b * r.V * r.Nv * r.Nu, r, row, vo, t);
}

// Row source of the filter kernel that rebins on the fly: filter row
// ((b * Vout + vo) * Nv + row), sample t.
template <typename TI>
struct RebinRows {
    const TI* in;
    RebinGrid r;
    __device__ __forceinline__ float operator()(int frow, int t) const {
        const int row = frow % r.Nv;
        const int vo = (frow / r.Nv) % r.Vout;
        const int b = frow / (r.Nv * r.Vout);
        return rebin_sample(in + (size_t)b * r.V * r.Nv * r.Nu, r, row, vo, t);
    }
};

}  // namespace xr
