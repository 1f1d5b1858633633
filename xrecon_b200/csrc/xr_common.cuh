// Shared device-side definitions of the B200 distance-driven projector.
//
// Geometry conventions follow the reference (XRecon include/types.h:35-119,
// include/xrmath.h:8-226): voxel centres at (i - N/2 + 1/2) d + shift with
// image row 0 at the top (+y), source at (-sin b, cos b) * SOD, detector
// boundaries mapped onto a common axis (x when cos^2 b > 1/2, else y), z
// mapped onto the axis plane by the magnification of the detector column
// centre (cells) and of the voxel line centre (voxels).
//
// Every operator of the path is the overlap kernel K[cell, voxel] with a
// diagonal scale on one side.  The kernels here evaluate K in normalised
// units: pixel positions along the current image line (one unit = one pixel)
// and voxel indices along z, in which
//     K = ovl_pos * ovl_zvox * dpix * dz * Mv(L)^2      (cone)
//     K = ovl_pos * ovl_zvox * dpix * dz                (3D parallel)
// where Mv(L) is the magnification of line L onto the axis.  The per-view
// geometry (boundary positions, column magnifications, cell scales) is set up
// in FP64 by xr_setup_views3d / xr_setup_views2d; the inner loops run in FP32
// on small local coordinates.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace xr {

// Device-wide sticky error word (one per device that loads the library).
// 0 = no error; kernels OR in a code when a bounded wait gives up (bits 0
// and 1) or, in builds with XR_DEBUG_BOUNDS, when an index checked by
// XR_BOUND falls outside its buffer (bit 2).  Defined here: the library is
// a single translation unit.
__device__ unsigned int g_device_error = 0;

constexpr unsigned XR_DEVERR_BOUNDS = 4u;

// XR_BOUND(i, lo, hi): the index i of a shared- or global-memory access.
// Release builds return i unchanged (the kernels' own arithmetic keeps every
// index inside its buffer).  Builds with XR_DEBUG_BOUNDS check it: an index
// outside [lo, hi] sets XR_DEVERR_BOUNDS in the error word and is clamped
// into the range, so the access stays in bounds and the kernel goes on; no
// check traps.
#ifdef XR_DEBUG_BOUNDS
__device__ __forceinline__ long long xr_check_index(long long i, long long lo, long long hi) {
    if (i < lo || i > hi) {
        atomicOr(&g_device_error, XR_DEVERR_BOUNDS);
        i = i < lo ? lo : hi;
    }
    return i;
}
#define XR_BOUND(i, lo, hi) (::xr::xr_check_index((i), (lo), (hi)))
#else
#define XR_BOUND(i, lo, hi) (i)
#endif

enum GeoType : int { GEO_PARALLEL = 0, GEO_FLAT = 1, GEO_ARC = 2 };
enum OpKind : int { OP_A = 0, OP_AT = 1, OP_B = 2, OP_BT = 3, OP_BW = 4, OP_BWT = 5 };
enum DType : int { DT_F32 = 0, DT_BF16 = 1, DT_F16 = 2 };

// Packed geometry; values are the reference's float32 options promoted to
// double (projector.py:106-110, projector3d.py:98-107).  2D uses Nz = Nv = 1.
struct Geom {
    int W, H, D, Nu, Nv, type;
    double dx, dy, dz, shx, shy, shz;
    double du, dv, shu, shv, sod, sdd;
};

// Per-view header (FP64 geometry, decisions taken like the reference CPU path).
struct ViewHdr {
    int use_x;      // common axis is x
    int keep;       // detector traversed in index order
    int nlines;     // H (use_x: lines are rows iy) or W (lines are columns ix)
    int npix;       // W or H: pixels along a line
    double beta, s, c;
    double sx, sy;          // source
    double spar, sperp;     // source coordinate along / across the axis
    double perpA, perpB;    // perpendicular coordinate of line L = perpA + perpB * L
    double q0, q1;          // 1 / Mv(L) = q0 + q1 * L   (1 for parallel)
    double dpix;            // pixel size along the line (dx or dy)
    float dcx, dcy;         // arc detector: central ray direction (column guesses)
    float sxf, syf;         // the source as the reference holds it in float32
};

// Per-view tables, structure of arrays, view-major.
//   pos_k(L) = bA[k] + bB[k] * L : position of detector boundary k (traversal
//              order) on line L in pixel units, k = 0..Nu
//   colQ[k]  = M_k / dz (3D), colR[k] = 1 / colQ[k] ; colE, colF, colM: cell scale of A,
//              s_A(k, r) = colE[k] * sqrt(colF[k] + (colM[k] * zc_r)^2)
// Per-view z placement and column scalars of a helical scan (all z measured
// from the view's source z), used by the kernels' HEL variants:
//   z0dz  = (volume bottom - source z) / dz
//   zd0   = lower boundary of detector row 0 - source z   (rows zd0 + r dv)
//   cw    = column width of B / B^T, sod' du'
//   zsrc  = source z (the projection's cell cosine takes the row's absolute z)
//   inv_du = 1 / du' (column guesses)
//   zlo, zhi = world z range, with a margin, of the voxels the view's detector
//          rows can reach anywhere in the image plane (views outside a voxel
//          run's z range are skipped)
//   zoffh = -zd0 / dv - 1/2 (row coordinate offset of the prefix gathers)
struct HelView {
    double z0dz, zd0, zoffh;
    float cw, zsrc, inv_du, pad;
    float zlo, zhi;
};

struct ViewTables {
    ViewHdr* hdr;
    double* bA;
    double* bB;
    double* colQ;
    double* colR;
    float* colE;
    float* colF;
    float* colM;
    HelView* hel;  // helical scans only, else null
    // circular arc detectors, voxel-driven operators (B, Bw and their
    // transposes) only, else null: two float4 per boundary k = 0..Nu of each
    // view, [2 (v (Nu + 1) + k)]: {float32 angle t, d(axis)/dt, dA, dB} and
    // {float32 axis position, tan(t) as a float pair hi + lo, 0}: the inputs
    // of the chained column walk (ArcChain); dA, dB are the boundary's line
    // coefficients minus those of boundary k - 1 (zero for k = 0), so the
    // walk's step to boundary k also reads column k - 1's width on line L,
    // dA + dB L pixels.
    float4* arc;
    // voxel gathers through the row prefix tables only, else null; per column
    // k of each view, [v Nu + k]: {dA, dB, R hi, R lo}: A and B of boundary
    // k + 1 minus those of boundary k in FP32 (the column's width on line L
    // is dA + dB L pixels), and colR as a float pair.  The gather evaluates
    // one boundary and one colR per (pixel, view) in FP64 and steps to the
    // neighbouring columns in FP32 from these.
    float4* colWR;
};

// ---------------------------------------------------------------- dtype io

template <typename T> __device__ __forceinline__ float ld(const T* p);
template <> __device__ __forceinline__ float ld<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p));
}
template <> __device__ __forceinline__ float ld<__half>(const __half* p) { return __half2float(__ldg(p)); }
// value conversions (registers, no load)
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }

template <typename T> __device__ __forceinline__ void st(T* p, float v);
template <> __device__ __forceinline__ void st<float>(float* p, float v) { *p = v; }
template <> __device__ __forceinline__ void st<__nv_bfloat16>(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ void st<__half>(__half* p, float v) { *p = __float2half_rn(v); }

// ---------------------------------------------------------------- geometry

// Axis decision and traversal order exactly as the reference CPU path takes
// them: float sin/cos of the float angle, cos^2 > 0.5 in float
// (src/cpu/forward3d.cpp:308-310, include/cpu3d_common.h:64-87).
__device__ __forceinline__ void view_decisions(float ang, int& use_x, int& keep) {
    const double a = (double)ang;
    const float cf = __double2float_rn(cos(a));
    const float sf = __double2float_rn(sin(a));
    use_x = __fmul_rn(cf, cf) > 0.5f;
    keep = use_x ? (cf >= 0.0f) : (sf >= 0.0f);
}

// Fill the per-view header.  On the device the axis decision is taken as the
// reference CPU path takes it (see view_decisions); on the host (only used
// for sizing staging windows) plain float arithmetic is used.
__host__ __device__ inline void make_view_hdr(const Geom& g, float ang, ViewHdr& h) {
#ifdef __CUDA_ARCH__
    view_decisions(ang, h.use_x, h.keep);
#else
    const float cf = (float)cos((double)ang), sf = (float)sin((double)ang);
    h.use_x = cf * cf > 0.5f;
    h.keep = h.use_x ? (cf >= 0.0f) : (sf >= 0.0f);
#endif
    h.beta = (double)ang;
    h.s = sin(h.beta);
    h.c = cos(h.beta);
    h.sx = -h.s * g.sod;
    h.sy = h.c * g.sod;
    h.spar = h.use_x ? h.sx : h.sy;
    h.sperp = h.use_x ? h.sy : h.sx;
    h.nlines = h.use_x ? g.H : g.W;
    h.npix = h.use_x ? g.W : g.H;
    if (h.use_x) { h.perpA = (0.5 * g.H - 0.5) * g.dy + g.shy; h.perpB = -g.dy; }
    else         { h.perpA = (0.5 - 0.5 * g.W) * g.dx + g.shx; h.perpB = g.dx; }
    if (g.type == GEO_PARALLEL) { h.q0 = 1.0; h.q1 = 0.0; }
    else { h.q0 = 1.0 - h.perpA / h.sperp; h.q1 = -h.perpB / h.sperp; }
    h.dpix = h.use_x ? g.dx : g.dy;
    h.dcx = (float)sin(h.beta + g.shu);
    h.dcy = (float)(-cos(h.beta + g.shu));
    // View2d.source = (-sinf(b) SOD, cosf(b) SOD) in float (xrmath.h:116-123)
    const float sodf = (float)g.sod;
#ifdef __CUDA_ARCH__
    h.sxf = __fmul_rn(-__double2float_rn(h.s), sodf);
    h.syf = __fmul_rn(__double2float_rn(h.c), sodf);
#else
    h.sxf = -(float)h.s * sodf;
    h.syf = (float)h.c * sodf;
#endif
}

// ------------------------------------------------ arc detector, float32

// Angle of arc boundary k (k + 1/2 for a column centre) as the reference
// forms it, every operation rounded to float32:
//     (k - Nu/2) du + shift_u + beta   (kept order),
//     (Nu/2 - k) du + shift_u + beta   (reversed)
// (src/cpu/forward3d.cpp:271-297, src/cpu/system_matrix2d.cpp:280-283,
// include/cpu3d_common.h:150-166).  The last sum rounds to a quantum of
// 4.8e-7 rad at |beta| ~ 2 pi, up to 5e-4 of a column at du = 1e-3, so the
// operator follows the rounded angle; everything after it is FP64.
__device__ __forceinline__ float arc_angle_f(const Geom& g, int keep, float kf, float ang) {
    const float half = __fmul_rn((float)g.Nu, 0.5f);
    const float sg = keep ? __fsub_rn(kf, half) : __fsub_rn(half, kf);
    return __fadd_rn(__fadd_rn(__fmul_rn(sg, (float)g.du), (float)g.shu), ang);
}

// Axis position of a ray at float angle t from the float source, as the
// reference computes it: src.x + src.y tan(t) on the x axis, src.y + src.x /
// tan(t) on the y axis, each step rounded to float32 (xrmath.h:24-38).  The
// sum cancels to about ulp(|src|), up to 1e-4 of a column near the 45-degree
// views, and the voxel-driven coefficients scale with it.  tf is tan(t)
// rounded to float (the C library's tanf of the reference's CPU path is
// within one unit of it).
__device__ __forceinline__ float arc_axis_f(const ViewHdr& h, float tf) {
    return h.use_x ? __fadd_rn(h.sxf, __fmul_rn(h.syf, tf)) : __fadd_rn(h.syf, __fdiv_rn(h.sxf, tf));
}

// Offset, on the common axis, of the boundary at the chained angle t from
// the direct boundary e = {t_d, tan hi, tan lo, axis} of the same index:
// tan(t) to float from tan(t_d + d) = T + d (1 + T^2)(1 + d T) + O(d^3),
// d = t - t_d (exact: both are floats a few units apart), then the float
// axis mapping.  Zero when t == t_d.
__device__ __forceinline__ float arc_chain_delta(const ViewHdr& h, const float4 e, float t) {
    const float d = __fsub_rn(t, e.x);
    const float S = fmaf(e.y, e.y, 1.0f);
    const float c = fmaf(d * S, fmaf(d, e.y, 1.0f), e.z);
    return __fsub_rn(arc_axis_f(h, __fadd_rn(e.y, c)), e.w);
}

// The column walk of a voxel-driven arc operator, chained in float32 as the
// reference walks it (include/cpu3d_common.h:160-196,
// src/cpu/backward2d.cpp:142-157): it starts at the column k0 holding the
// voxel's first edge, at that column's lower angle (detector kept in order)
// or at the next column's angle plus du (reversed), and each further
// boundary angle is the previous one plus du (kept) or minus du (reversed).
// The step to boundary j returns its axis offset from the direct boundary:
//   next_exact:  the float axis mapping of the chained angle (arc_chain_delta);
//   next_linear: (t - t_j) d(axis)/dt at the direct angle t_j.
// The chained angle drifts from the direct one by the accumulated roundings
// (several float units after a few columns), which the reference's results
// carry.  The voxel-owned gathers (B, Bw) take the linear step: it leaves
// out only the float rounding of the chained axis positions, which their
// sums over columns and views average away (within 4e-6 of the reference
// where the exact step is within 3.9e-6); the cell-owned transposes, which
// do not average it, take the exact step.
struct ArcChain {
    float t, step;
    // e: the view's arc entries (two float4 per boundary)
    __device__ __forceinline__ void start(const float4* __restrict__ e, int k0, int keep, float du) {
        step = keep ? du : -du;
        t = keep ? e[2 * k0].x : __fadd_rn(e[2 * (k0 + 1)].x, du);
    }
    __device__ __forceinline__ float next_linear(const float4* __restrict__ e, int j) {
        t = __fadd_rn(t, step);
        const float4 a = e[2 * j];
        return __fsub_rn(t, a.x) * a.y;
    }
    // the same, and the width of column j - 1 on line Lf (pixels)
    __device__ __forceinline__ float next_linear(const float4* __restrict__ e, int j, float Lf, float& width) {
        t = __fadd_rn(t, step);
        const float4 a = e[2 * j];
        width = fmaf(a.w, Lf, a.z);
        return __fsub_rn(t, a.x) * a.y;
    }
    __device__ __forceinline__ float next_exact(const ViewHdr& h, const float4* __restrict__ e, int j) {
        t = __fadd_rn(t, step);
        const float4 a = e[2 * j], b = e[2 * j + 1];
        return arc_chain_delta(h, make_float4(a.x, b.y, b.z, b.x), t);
    }
};

// Column-centre z magnification M_k onto the axis plane (forward3d.cpp:258-297).
__host__ __device__ inline double column_mag(const Geom& g, const ViewHdr& h, int k, double uscale) {
    if (g.type == GEO_PARALLEL) return 1.0;
    const double sgc = (h.keep ? ((double)k + 0.5 - 0.5 * g.Nu) : (0.5 * g.Nu - (double)k - 0.5));
    double cx, cy;
    if (g.type == GEO_FLAT) {
        const double u = (sgc * g.du + g.shu) * uscale;
        cx = u * h.c;
        cy = u * h.s;
    } else {
        const double ac = sgc * g.du + g.shu + h.beta;
        cx = sin(ac) * g.sdd + h.sx;
        cy = -cos(ac) * g.sdd + h.sy;
    }
    return h.use_x ? h.sy / (h.sy - cy) : h.sx / (h.sx - cx);
}

__host__ __device__ __forceinline__ double sigma(int keep, double k, int nu) {
    return keep ? (k - 0.5 * nu) : (0.5 * nu - k);
}

// Intercept of the ray source -> point with the common axis (xrmath.h:8-22).
__host__ __device__ __forceinline__ double map_point(const ViewHdr& h, double px, double py) {
    if (h.use_x) return (h.sx * py - h.sy * px) / (py - h.sy);
    return (h.sy * px - h.sx * py) / (px - h.sx);
}

// Same for a ray leaving the source at angle a (xrmath.h:24-38).
__host__ __device__ __forceinline__ double map_angle(const ViewHdr& h, double a) {
    if (h.use_x) return h.sx + h.sy * tan(a);
    return h.sy + h.sx / tan(a);
}

// Axis coordinate of detector boundary k (traversal order).
//   flat: forward3d.cpp:229-243 (3D scales u by SOD/SDD; 2D du is already
//         the isocentre spacing, projector.py:97) ; arc: forward3d.cpp:271-283 ;
//   parallel: forward3d.cpp:53-56.
__host__ __device__ __forceinline__ double boundary_axis(const Geom& g, const ViewHdr& h, double k, double uscale) {
    const double sg = sigma(h.keep, k, g.Nu);
    if (g.type == GEO_FLAT) {
        const double u = (sg * g.du + g.shu) * uscale;
        return map_point(h, u * h.c, u * h.s);
    }
    if (g.type == GEO_ARC) return map_angle(h, sg * g.du + g.shu + h.beta);
    const double u = sg * g.du + g.shu;
    return h.use_x ? u / h.c : u / h.s;
}

// Line-position coefficients of the ray through axis point D:
// pos(L) = A + B * L in pixel units along line L.
__host__ __device__ __forceinline__ void boundary_line_coeffs(const Geom& g, const ViewHdr& h, double D,
                                                     double& A, double& B) {
    if (h.use_x) {
        const double pyA = (0.5 * g.H - 0.5) * g.dy + g.shy, pyB = -g.dy;
        const double x0 = -0.5 * g.W * g.dx + g.shx;
        if (g.type == GEO_PARALLEL) {
            const double t = h.s / h.c;
            A = (D - t * pyA - x0) / g.dx;
            B = -t * pyB / g.dx;
        } else {
            const double e = D - h.sx;
            A = (h.sx + e * (1.0 - pyA / h.sy) - x0) / g.dx;
            B = -e * pyB / (h.sy * g.dx);
        }
    } else {
        const double pxA = (0.5 - 0.5 * g.W) * g.dx + g.shx, pxB = g.dx;
        const double y0 = -0.5 * g.H * g.dy + g.shy;
        if (g.type == GEO_PARALLEL) {
            const double t = h.c / h.s;
            A = (D - t * pxA - y0) / g.dy;
            B = -t * pxB / g.dy;
        } else {
            const double e = D - h.sy;
            A = (h.sy + e * (1.0 - pxA / h.sx) - y0) / g.dy;
            B = -e * pxB / (h.sx * g.dy);
        }
    }
}

// atan2 for column guesses only: an odd polynomial x P(x^2) of degree 11,
// least-squares fitted to atan on [0, 1] for this library (max error 2.0e-6
// rad in FP32), with the usual octant reduction.  Callers widen their column
// bracket by the error over the angular column width.
__device__ __forceinline__ float guess_atan2f(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    const float t = mx > 0.0f ? __fdividef(mn, mx) : 0.0f;
    const float t2 = t * t;
    float p = -0.01175929419696331f;
    p = fmaf(p, t2, 0.05272875353693962f);
    p = fmaf(p, t2, -0.11647544801235199f);
    p = fmaf(p, t2, 0.19354581832885742f);
    p = fmaf(p, t2, -0.3326205611228943f);
    p = fmaf(p, t2, 0.9999769330024719f);
    float r = t * p;
    if (ay > ax) r = 1.5707963267948966f - r;
    if (x < 0.0f) r = 3.141592653589793f - r;
    return y < 0.0f ? -r : r;
}
constexpr float XR_GUESS_ATAN_ERR = 4.0e-6f;  // bound used to widen brackets

// Fractional traversal index of the detector position hit by the ray
// source -> world point (x, y).  FP32 guess only; callers verify against the
// FP64 boundary tables.
__device__ __forceinline__ float col_guess(const Geom& g, const ViewHdr& h, float x, float y, float uscale) {
    const float s = (float)h.s, c = (float)h.c;
    float sg;
    if (g.type == GEO_FLAT) {
        const float R = (float)g.sod;
        const float u = R * (x * c + y * s) / (R + x * s - y * c);   // virtual detector coordinate
        sg = (u / uscale - (float)g.shu) / (float)g.du;
    } else if (g.type == GEO_ARC) {
        const float ac = (float)(h.beta + g.shu);
        const float dcx = sinf(ac), dcy = -cosf(ac);
        const float ex = x - (float)h.sx, ey = y - (float)h.sy;
        const float gam = atan2f(dcx * ey - dcy * ex, dcx * ex + dcy * ey);
        sg = gam / (float)g.du;
    } else {
        const float u = x * c + y * s;
        sg = (u - (float)g.shu) / (float)g.du;
    }
    return h.keep ? sg + 0.5f * g.Nu : 0.5f * g.Nu - sg;
}

// World coordinates of pixel boundary `p` (pixel units) on line L.
__device__ __forceinline__ void line_point(const Geom& g, const ViewHdr& h, int L, float p,
                                           float& x, float& y) {
    if (h.use_x) {
        y = (float)((0.5 * g.H - L - 0.5) * g.dy + g.shy);
        x = (float)(-0.5 * g.W * g.dx + g.shx) + p * (float)g.dx;
    } else {
        x = (float)((L - 0.5 * g.W + 0.5) * g.dx + g.shx);
        y = (float)(-0.5 * g.H * g.dy + g.shy) + p * (float)g.dy;
    }
}

// FBP voxel weight: cone_voxel_weight_flat / _arc (xrmath.h:215-226,
// backward2d.cpp:93 / :161).
__device__ __forceinline__ float fbp_weight(const Geom& g, const ViewHdr& h, float px, float py) {
    if (g.type == GEO_FLAT) {
        const float R = (float)g.sod;
        const float d = __fdividef((float)h.sx * px + (float)h.sy * py, R);
        const float den = R - d;
        return __fdividef(R * R, den * den);
    }
    if (g.type == GEO_ARC) {
        const float ex = (float)h.sx - px, ey = (float)h.sy - py;
        return __fdividef(1.0f, ex * ex + ey * ey);
    }
    return 1.0f;
}

// Voxel-centre world coordinates of pixel index p (pixel units, integer) on line L.
__device__ __forceinline__ void pixel_center(const Geom& g, const ViewHdr& h, int L, int p,
                                             float& px, float& py) {
    int ix, iy;
    if (h.use_x) { ix = p; iy = L; } else { ix = L; iy = g.H - 1 - p; }
    px = (float)((ix - 0.5 * g.W + 0.5) * g.dx + g.shx);
    py = (float)((0.5 * g.H - iy - 0.5) * g.dy + g.shy);
}

}  // namespace xr
