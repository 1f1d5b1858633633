// Helical cone-beam scans with an arc detector (the reference's
// src/kernels/helical_arc3d.cu, bound at src/api/torch_binding.cpp:525-612).
//
// Every view has its own source placement, source_pos[4][V] =
// (source_z, shift_radius, shift_angle, shift_z), helical_arc3d.cu:382-395:
//     sod' = SOD + sr, sdd' = SDD + sr, du' = du SDD / sdd',
//     shu' = shu SDD / sdd' - sa (sdd' - sod') / sdd',
//     source at angle beta + sa, column angles sg du' + shu' + beta,
//     source z = source_z + shift_z, detector rows (r - Nv/2) dv + source_z + shv.
// A, A^T, B, B^T are the cone-arc DD operators of the circular path with
// these per-view values: setup_views_helical_kernel writes the usual view
// tables from a per-view Geom, plus a HelView with the view's z placement,
// and the kernels' HEL variants read it.  The reference's A takes the cell
// cosine with the row's absolute z (helical_arc3d.cu:432), which the HEL
// variants reproduce.
//
// Bw and Bw^T (helical_arc3d.cu:1112-1505) weight each (voxel, view) pair of
// the voxel's view window (a span of views centred on the view whose source
// z is the voxel's z) with a redundancy weight and scale each voxel by
// (pi / |dbeta|) / (sum of the weights of the views whose detector its centre
// hits), clamped to [1/32, 32].  The window, the weights and the "measured"
// test are evaluated in FP32 with the reference's operation order (explicit
// round-to-nearest intrinsics where the result feeds a discrete decision), the
// DD footprint through the FP64 view tables as elsewhere:
//   hel_zwin_kernel   per z slice: window [vs, ve], its end angles, centre
//                     angle, and whether its weights depend on the view alone
//   hel_wtab_kernel   the weights of those slices, per (slice, view)
//   hel_wbp_kernel    Bw: voxel gather over the run's window through the row
//                     prefix tables (xr_vox_prefix.cuh), per-voxel weights and
//                     normalisation in one pass; its DD-free form gives the
//                     normalisation volume that Bw^T needs
//   hel_wbpt_kernel   Bw^T: cell gather, per-voxel weights
#pragma once

#include "xr_vox_prefix.cuh"

namespace xr {

struct HelOpts {
    int view_mode;    // 0 auto (from the pitch), 1 half scan, 2 one turn, 3 fixed turns
    int weight_mode;  // 0 conjugate-ray redundancy ("2d"), 1 tangential ("tang3d")
    float view_turns, halfscan_coef, tang_k, tang_blend;
};

// Per-view FP32 scalars of the weighted kernels (helical_arc3d.cu:1148-1160).
struct HelWView {
    float sod, sdd, du, shu, beta, sinv, cosv, sx, sy, szv, zs, shz;
    float inv_du, pad0, pad1, pad2;  // 1 / du (fast pre-tests only)
};

// Per z slice: view window [vs, ve], its end angles, the centre angle, the
// slice's z, and whether the slice's weights depend on the view alone (the
// conjugate-ray weight of a window spanning a full turn), in which case they
// are tabulated per (slice, view) once per call.
struct HelZ {
    int vs, ve;
    float bs, be, bc, pz;
    int full, pad;
};

constexpr float XR_PI_F = 3.14159265358979323846f;

// Scan scalars of the weighted kernels: mean angle step (angles[V-1] -
// angles[0]) / (V - 1), half fan angle du (Nu - 1) / 2, column width SOD du.
// Written on the device by hel_zwin_kernel (the angles live there).
struct HelScanF {
    float db, gmax, cwW, pad;
};

// ----------------------------------------------------------------- setup

// One thread per (view, boundary k = 0..Nu), as setup_views_kernel, with the
// view's own Geom; thread k == 0 also writes the view's HelView / HelWView.
__global__ void setup_views_helical_kernel(const Geom g, const float* __restrict__ ang,
                                           const float* __restrict__ sp, const int nview, const ViewTables vt,
                                           HelWView* __restrict__ wv) {
    const int v = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nview || k > g.Nu) return;
    const float zs = sp[v], sr = sp[nview + v], sa = sp[2 * nview + v], szs = sp[3 * nview + v];
    const float SOD = (float)g.sod, SDD = (float)g.sdd;
    const float sod = __fadd_rn(SOD, sr), sdd = __fadd_rn(SDD, sr);
    const float du = __fdiv_rn(__fmul_rn((float)g.du, SDD), sdd);
    const float shu = __fsub_rn(__fdiv_rn(__fmul_rn((float)g.shu, SDD), sdd),
                                __fdiv_rn(__fmul_rn(sa, __fsub_rn(sdd, sod)), sdd));
    const float beta = __fadd_rn(ang[v], sa);
    const float zsrc = __fadd_rn(zs, szs);
    Geom gv = g;
    gv.sod = sod;
    gv.sdd = sdd;
    gv.du = du;
    // column angle sg du' + shu' + beta_unshifted, relative to the source angle
    gv.shu = (double)shu + ((double)ang[v] - (double)beta);
    setup_view_entry(gv, 1, beta, v, k, vt);
    if (k != 0) return;
    HelView hv;
    hv.zd0 = -0.5 * g.Nv * g.dv + (double)zs + g.shv - (double)zsrc;
    hv.z0dz = (-0.5 * g.D * g.dz + g.shz - (double)zsrc) / g.dz;
    hv.zoffh = -hv.zd0 / g.dv - 0.5;  // arc rows: dvv = dv
    hv.cw = __fmul_rn(sod, du);
    hv.zsrc = zsrc;
    hv.inv_du = (float)(1.0 / (double)du);
    hv.pad = 0.0f;
    {
        // A voxel at in-plane distance r from the source sees detector row
        // z (relative to the source) at z_vox = z_row r / sdd'.  r spans
        // sod' -+ the image half-diagonal; 2 % on r and two voxels of margin
        // keep the range conservative for the DD footprints.
        const double hx = 0.5 * g.W * g.dx + fabs(g.shx), hy = 0.5 * g.H * g.dy + fabs(g.shy);
        const double rxy = sqrt(hx * hx + hy * hy);
        const double rmin = fmax(0.98 * ((double)sod - rxy), 0.0), rmax = 1.02 * ((double)sod + rxy);
        const double zb0 = hv.zd0, zb1 = hv.zd0 + g.Nv * g.dv;
        const double lo = fmin(zb0 * rmin, zb0 * rmax) / (double)sdd;
        const double hi = fmax(zb1 * rmin, zb1 * rmax) / (double)sdd;
        hv.zlo = (float)((double)zsrc + lo - 2.0 * g.dz);
        hv.zhi = (float)((double)zsrc + hi + 2.0 * g.dz);
    }
    vt.hel[v] = hv;
    HelWView w;
    w.sod = sod;
    w.sdd = sdd;
    w.du = du;
    w.shu = shu;
    w.beta = beta;
    w.sinv = sinf(beta);
    w.cosv = cosf(beta);
    w.sx = __fmul_rn(-w.sinv, sod);
    w.sy = __fmul_rn(w.cosv, sod);
    w.szv = zsrc;
    w.zs = zs;
    w.shz = szs;
    w.inv_du = (float)(1.0 / (double)du);
    w.pad0 = w.pad1 = w.pad2 = 0.0f;
    wv[v] = w;
}

// ---------------------------------------------------------------- weights

__device__ __forceinline__ float hw_clamp_unit(float x) { return fminf(1.0f, fmaxf(0.0f, x)); }

__device__ __forceinline__ float hw_smooth_step(float x) {
    x = hw_clamp_unit(x);
    return 0.5f * (1.0f - cosf(XR_PI_F * x));
}

__device__ __forceinline__ float hw_window_quality(float beta, float bs, float be, float gamma, float gmax) {
    const float lo = fminf(bs, be), hi = fmaxf(bs, be);
    if (beta < lo || beta > hi) return 0.0f;
    const float gc = fminf(fmaxf(gamma, -gmax), gmax);
    const float lw = fmaxf(1.0e-6f, 2.0f * (gmax - gc));
    const float rw = fmaxf(1.0e-6f, 2.0f * (gmax + gc));
    if (beta < __fadd_rn(lo, lw)) return hw_smooth_step(__fdiv_rn(beta - lo, lw));
    if (beta > __fsub_rn(hi, rw)) return hw_smooth_step(__fdiv_rn(hi - beta, rw));
    return 1.0f;
}

__device__ __forceinline__ float hw_center_turn(float beta, float bc, float bs, float be, float db) {
    const float lo = fminf(bs, be), hi = fmaxf(bs, be);
    if (beta < lo || beta > hi) return 0.0f;
    const float adb = fmaxf(fabsf(db), 1.0e-6f);
    const float half = 0.5f * (hi - lo);
    const float dist = fabsf(beta - bc);
    const float crad = fminf(XR_PI_F, half);
    if (dist <= crad) return 1.0f;
    const float ow = fmaxf(half - crad, 4.0f * adb);
    return hw_smooth_step(__fdiv_rn(half - dist, ow));
}

__device__ __forceinline__ float hw_source_z_at(float beta, const float* __restrict__ ang,
                                                const float* __restrict__ zsrc, int nview) {
    if (nview <= 1) return zsrc[0];
    const float a0 = ang[0], a1 = ang[nview - 1];
    const float range = a1 - a0;
    if (fabsf(range) <= 1.0e-6f) return zsrc[0];
    const float dzdb = __fdiv_rn(zsrc[nview - 1] - zsrc[0], range);
    return __fadd_rn(zsrc[0], __fmul_rn(beta - a0, dzdb));
}

__device__ __forceinline__ float hw_edge_taper(float beta, float bc, float bs, float be, float db) {
    const float lo = fminf(bs, be), hi = fmaxf(bs, be);
    if (beta < lo || beta > hi) return 0.0f;
    const float span = hi - lo, half = 0.5f * span;
    if (span <= __fadd_rn(XR_PI_F, __fmul_rn(8.0f, fabsf(db)))) return 1.0f;
    const float crad = fminf(XR_PI_F, half);
    const float dist = fabsf(beta - bc);
    if (dist <= crad) return 1.0f;
    const float ew = fmaxf(half - crad, 4.0f * fabsf(db));
    return hw_smooth_step(__fdiv_rn(half - dist, ew));
}

// helical_arc3d.cu:212-241
__device__ __forceinline__ float hw_conjugate(float beta, float gamma, float bc, float bs, float be, float db,
                                              float gmax) {
    const float span = fabsf(be - bs);
    const float adb = fmaxf(fabsf(db), 1.0e-6f);
    if (span >= __fsub_rn(2.0f * XR_PI_F, 2.0f * adb)) {
        const float turns = fmaxf(1.0f, floorf(__fdiv_rn(__fadd_rn(span, 2.0f * adb), 2.0f * XR_PI_F)));
        return __fdiv_rn(0.5f * hw_center_turn(beta, bc, bs, be, db), turns);
    }
    const float q = hw_window_quality(beta, bs, be, gamma, gmax);
    if (q <= 0.0f) return 0.0f;
    const float dir = (db >= 0.0f) ? 1.0f : -1.0f;
    float den = 0.0f;
    for (int k = -4; k <= 4; ++k) {
        const float turn = dir * 2.0f * XR_PI_F * (float)k;
        den += hw_window_quality(__fadd_rn(beta, turn), bs, be, gamma, gmax);
        const float bcj = __fadd_rn(__fadd_rn(beta, __fmul_rn(dir, __fadd_rn(XR_PI_F, 2.0f * gamma))), turn);
        den += hw_window_quality(bcj, bs, be, -gamma, gmax);
    }
    return __fdiv_rn(q, fmaxf(den, 1.0e-6f));
}

// Redundancy weight of one (voxel, view) pair, helical_arc3d.cu:243-303.
__device__ __forceinline__ float hw_weight(const HelOpts& o, const Geom& g, float px, float py, float pz, float beta,
                                          float gamma, float src_z, float ray_xy, float bc, float bs, float be,
                                          float db, float gmax, const float* __restrict__ ang,
                                          const float* __restrict__ zsrc, int nview) {
    if (o.weight_mode == 0) return hw_conjugate(beta, gamma, bc, bs, be, db, gmax);
    const float span = fabsf(be - bs);
    const float dir = (beta < bc) ? 1.0f : -1.0f;
    const float bcj = __fadd_rn(beta, __fmul_rn(dir, __fadd_rn(XR_PI_F, 2.0f * gamma)));
    float dq, cq;
    if (span < __fsub_rn(2.0f * XR_PI_F, 2.0f * fabsf(db))) {
        dq = hw_window_quality(beta, bs, be, gamma, gmax);
        cq = hw_window_quality(bcj, bs, be, -gamma, gmax);
    } else {
        dq = hw_edge_taper(beta, bc, bs, be, db);
        cq = hw_edge_taper(bcj, bc, bs, be, db);
    }
    if (dq <= 0.0f) return 0.0f;
    if (cq <= 0.0f) return 1.0f;
    const float zc = hw_source_z_at(bcj, ang, zsrc, nview);
    const float SOD = (float)g.sod;
    const float sxc = -sinf(bcj) * SOD, syc = cosf(bcj) * SOD;
    const float rxc = px - sxc, ryc = py - syc;
    const float rxyc = sqrtf(rxc * rxc + ryc * ryc);
    const float ta = __fdiv_rn(fabsf(pz - src_z), fmaxf(ray_xy, 1.0e-6f));
    const float tac = __fdiv_rn(fabsf(pz - zc), fmaxf(rxyc, 1.0e-6f));
    const float kk = fminf(fmaxf(o.tang_k, 0.0f), 32.0f);
    const float gg = powf(fmaxf(ta, 1.0e-6f), kk);
    const float ggc = powf(fmaxf(tac, 1.0e-6f), kk);
    const float w2 = __fdiv_rn(dq, fmaxf(dq + cq, 1.0e-6f));
    const float den = dq * ggc + cq * gg;
    const float w3 = __fdiv_rn(dq * ggc, fmaxf(den, 1.0e-6f));
    const float blend = hw_clamp_unit(o.tang_blend);
    return (1.0f - blend) * w2 + blend * w3;
}

// Voxel centre in world coordinates, helical_arc3d.cu:1130-1132.
__device__ __forceinline__ float hw_px(const Geom& g, int ix) {
    return __fadd_rn(__fmul_rn(__fadd_rn(__fsub_rn((float)ix, __fdiv_rn((float)g.W, 2.0f)), 0.5f), (float)g.dx),
                     (float)g.shx);
}
__device__ __forceinline__ float hw_py(const Geom& g, int iy) {
    return __fadd_rn(__fmul_rn(__fsub_rn(__fsub_rn(__fmul_rn((float)g.H, 0.5f), (float)iy), 0.5f), (float)g.dy),
                     (float)g.shy);
}
__device__ __forceinline__ float hw_pz(const Geom& g, int iz) {
    return __fadd_rn(__fmul_rn(__fadd_rn(__fsub_rn((float)iz, __fdiv_rn((float)g.D, 2.0f)), 0.5f), (float)g.dz),
                     (float)g.shz);
}

// Fan angle of the voxel centre in this view and the ray's length in xy
// (helical_arc3d.cu:1161-1166).
__device__ __forceinline__ void hw_ray(const HelWView& w, float px, float py, float& gamma, float& rxy,
                                       float& rx, float& ry) {
    rx = __fsub_rn(px, w.sx);
    ry = __fsub_rn(py, w.sy);
    rxy = sqrtf(__fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)));
    const float xb = __fsub_rn(__fmul_rn(w.cosv, px), __fmul_rn(w.sinv, py));
    const float yb = __fadd_rn(__fmul_rn(w.sinv, px), __fmul_rn(w.cosv, py));
    gamma = atan2f(yb, __fsub_rn(w.sod, xb));
}

// Does the ray through the voxel centre hit the detector?
// helical_arc3d.cu:305-336, split into the column test (per pixel and view)
// and the row test (per voxel), with gamma and the xy ray length as hw_ray
// gives them.
__device__ __forceinline__ bool hw_col_in(const Geom& g, const HelWView& w, float gamma) {
    const float col = __fsub_rn(__fadd_rn(__fdiv_rn(__fsub_rn(gamma, w.shu), w.du), __fmul_rn((float)g.Nu, 0.5f)),
                                0.5f);
    return !(col < -0.5f || col > __fsub_rn((float)g.Nu, 0.5f));
}
__device__ __forceinline__ bool hw_row_in(const Geom& g, const HelWView& w, float rxy, float pz) {
    const float det_z = __fadd_rn(w.szv, __fdiv_rn(__fmul_rn(w.sdd, __fsub_rn(pz, w.szv)), rxy));
    const float row = __fsub_rn(__fadd_rn(__fdiv_rn(__fsub_rn(__fsub_rn(det_z, w.zs), (float)g.shv), (float)g.dv),
                                          __fmul_rn((float)g.Nv, 0.5f)),
                                0.5f);
    return row >= -0.5f && row <= __fsub_rn((float)g.Nv, 0.5f);
}

// The same two tests decided from cheap approximations (reciprocals, the
// fitted atan2 of the column guesses), falling back to the exact forms above
// only when the approximate row or column lies within a safety band of an
// edge: the approximations differ from the exact FP32 values by far less
// than the band (the atan2 fit by XR_GUESS_ATAN_ERR rad, the rest by a few
// ulps of values below 2^13), so every decision equals the exact one.
constexpr float HW_BAND = 1.0e-3f;

__device__ __forceinline__ bool hw_col_in_fast(const Geom& g, const HelWView& w, float px, float py, float xb,
                                               float yb) {
    const float ga = guess_atan2f(yb, w.sod - xb);
    const float col = (ga - w.shu) * w.inv_du + 0.5f * (float)g.Nu - 0.5f;
    const float band = HW_BAND + XR_GUESS_ATAN_ERR * w.inv_du;
    const float top = (float)g.Nu - 0.5f;
    if (col > -0.5f + band && col < top - band) return true;
    if (col < -0.5f - band || col > top + band) return false;
    const float xe = __fsub_rn(__fmul_rn(w.cosv, px), __fmul_rn(w.sinv, py));
    const float ye = __fadd_rn(__fmul_rn(w.sinv, px), __fmul_rn(w.cosv, py));
    return hw_col_in(g, w, atan2f(ye, __fsub_rn(w.sod, xe)));
}

// tz = sdd / rxy (approximate), inv_dv = 1 / dv
__device__ __forceinline__ bool hw_row_in_fast(const Geom& g, const HelWView& w, float rxy, float tz, float inv_dv,
                                               float pz) {
    const float row = (w.szv + (pz - w.szv) * tz - w.zs - (float)g.shv) * inv_dv + 0.5f * (float)g.Nv - 0.5f;
    const float top = (float)g.Nv - 0.5f;
    if (row > -0.5f + HW_BAND && row < top - HW_BAND) return true;
    if (row < -0.5f - HW_BAND || row > top + HW_BAND) return false;
    return hw_row_in(g, w, rxy, pz);
}

// ------------------------------------------------------------ view windows

// helical_arc3d.cu:141-210 and :121-139, one thread per z slice; thread 0
// also writes the scan scalars.
__global__ void hel_zwin_kernel(const Geom g, const HelOpts o, const float* __restrict__ ang,
                                const float* __restrict__ zsrc, const int nview, HelZ* __restrict__ zw,
                                HelScanF* __restrict__ scan) {
    const int iz = blockIdx.x * blockDim.x + threadIdx.x;
    if (iz == 0) {
        HelScanF sc;
        sc.db = (nview > 1) ? __fdiv_rn(__fsub_rn(ang[nview - 1], ang[0]), (float)(nview - 1)) : 0.0f;
        sc.gmax = __fmul_rn(__fmul_rn((float)g.du, (float)(g.Nu - 1)), 0.5f);
        sc.cwW = __fmul_rn((float)g.sod, (float)g.du);
        sc.pad = 0.0f;
        *scan = sc;
    }
    if (iz >= g.D) return;
    const float pz = hw_pz(g, iz);
    int vs = 0, ve = 0;
    if (nview > 1) {
        const float a0 = ang[0], a1 = ang[nview - 1], z0 = zsrc[0], z1 = zsrc[nview - 1];
        const float range = __fsub_rn(a1, a0);
        if (fabsf(range) < 1.0e-6f) {
            ve = nview - 1;
        } else {
            const float db = __fdiv_rn(range, fmaxf(1.0f, (float)(nview - 1)));
            const float dzdb = __fdiv_rn(__fsub_rn(z1, z0), range);
            if (fabsf(db) < 1.0e-8f || fabsf(dzdb) < 1.0e-8f) {
                ve = nview - 1;
            } else {
                const float du = (float)g.du, dv = (float)g.dv, SOD = (float)g.sod, SDD = (float)g.sdd;
                const float gmax = __fmul_rn(__fmul_rn(du, (float)(g.Nu - 1)), 0.5f);
                const float half_scan = __fmul_rn(__fadd_rn(XR_PI_F, __fmul_rn(2.0f, gmax)),
                                                  fmaxf(o.halfscan_coef, 1.0f));
                float span = 2.0f * XR_PI_F;
                if (o.view_mode == 1) span = half_scan;
                else if (o.view_mode == 2) span = 2.0f * XR_PI_F;
                else if (o.view_mode == 3) span = __fmul_rn(__fmul_rn(fmaxf(0.25f, o.view_turns), 2.0f), XR_PI_F);
                else {
                    const float ppt = __fmul_rn(__fmul_rn(fabsf(dzdb), 2.0f), XR_PI_F);
                    const float iso_h = fmaxf(__fdiv_rn(__fmul_rn(__fmul_rn(dv, (float)g.Nv), SOD), SDD), dv);
                    const float np = __fdiv_rn(ppt, fmaxf(iso_h, 1.0e-6f));
                    if (np >= 1.25f) span = half_scan;
                    else if (np >= 0.45f) span = 2.0f * XR_PI_F;
                    else if (np >= 0.25f) span = 3.0f * XR_PI_F;
                    else span = 5.0f * XR_PI_F;
                }
                // A window of V or more views is all views, and a centre
                // beyond +-4V gives the same clamped window as +-4V: both
                // bounds keep the integer arithmetic below in range.
                const float nwf = ceilf(__fdiv_rn(span, fabsf(db)));
                const int nwin = (nwf >= (float)nview) ? nview : (nwf < 1.0f ? 1 : (int)nwf);
                const float bc = __fadd_rn(a0, __fdiv_rn(__fsub_rn(pz, z0), dzdb));
                const float vcf = roundf(__fdiv_rn(__fsub_rn(bc, a0), db));
                const int vc = (int)fminf(fmaxf(vcf, -4.0f * (float)nview), 4.0f * (float)nview);
                vs = max(0, vc - nwin / 2);
                ve = min(nview - 1, vs + nwin - 1);
                vs = max(0, ve - nwin + 1);
            }
        }
    }
    HelZ z;
    z.vs = vs;
    z.ve = ve;
    z.bs = ang[vs];
    z.be = ang[ve];
    z.pz = pz;
    // centre angle, helical_arc3d.cu:121-139
    float bc;
    if (nview <= 1) {
        bc = 0.5f * (z.bs + z.be);
    } else {
        const float a0 = ang[0], a1 = ang[nview - 1], z0 = zsrc[0], z1 = zsrc[nview - 1];
        const float range = __fsub_rn(a1, a0);
        const float dzdb = (fabsf(range) > 1.0e-6f) ? __fdiv_rn(__fsub_rn(z1, z0), range) : 0.0f;
        if (fabsf(dzdb) <= 1.0e-8f) {
            bc = 0.5f * (z.bs + z.be);
        } else {
            const float b = __fadd_rn(a0, __fdiv_rn(__fsub_rn(pz, z0), dzdb));
            bc = fminf(fmaxf(b, fminf(z.bs, z.be)), fmaxf(z.bs, z.be));
        }
    }
    z.bc = bc;
    {
        // hw_conjugate's full-turn branch (no fan angle, no voxel position)
        const float db = (nview > 1) ? __fdiv_rn(__fsub_rn(ang[nview - 1], ang[0]), (float)(nview - 1)) : 0.0f;
        const float adb = fmaxf(fabsf(db), 1.0e-6f);
        z.full = (o.weight_mode == 0) && (fabsf(z.be - z.bs) >= __fsub_rn(2.0f * XR_PI_F, 2.0f * adb));
    }
    z.pad = 0;
    zw[iz] = z;
}

// Weight table of the full-turn slices, rows for slices -1 .. D + 1:
// wtab[(iz + 1) * nview + v], zero outside the slice's window, for the other
// slices and for the three slices outside the volume (which the TMA cell
// gather's staged window and look-ahead reach).
__global__ void hel_wtab_kernel(const HelScanF* __restrict__ scan, const HelWView* __restrict__ wv,
                                const HelZ* __restrict__ zw, const int D, const int nview, float* __restrict__ wtab) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = (int)blockIdx.y - 1;
    if (v >= nview) return;
    float w = 0.0f;
    if (iz >= 0 && iz < D) {
        const HelZ z = zw[iz];
        if (z.full && v >= z.vs && v <= z.ve) {
            const HelScanF s = *scan;
            w = hw_conjugate(wv[v].beta, 0.0f, z.bc, z.bs, z.be, s.db, s.gmax);
        }
    }
    wtab[(size_t)(iz + 1) * nview + v] = w;
}

// ---------------------------------------------------------------------- Bw

// Voxel gather of the weighted backprojection, with the per-voxel
// normalisation in the same pass.  CTA = 32 x NWY pixels of the image plane
// times a run of R z slices (the run's windows are CTA-uniform); the view
// loop covers the union of the run's windows.  Per (pixel, view) the fan
// angle and ray length are computed once; per voxel of the run the weight
// comes from the slice table (full-turn slices) or is evaluated, and is
// summed into the voxel's normalisation when the ray through its centre
// hits the detector (helical_arc3d.cu:1141-1180).  The z integral of a
// (voxel, column) pair comes from the row prefix table of the view
// (xr_vox_prefix.cuh) as in vox_prefix3d_kernel.
//   DD true : out = Bw voxels, (pi / |dbeta|) / sum, clamped, times the sum
//             of the weighted footprints
//   DD false: out = the normalisation itself (for Bw^T); no footprints
#ifndef XR_HWBP_MINB
#define XR_HWBP_MINB 4  // CTAs per SM the register budget is sized for
#endif
template <int R, int NWY, bool DD>
__global__ void __launch_bounds__(32 * NWY, XR_HWBP_MINB)
hel_wbp_kernel(const Geom g, const GeomF gf, const ViewTables vt, const HelOpts o, const HelScanF* __restrict__ scan,
               const HelWView* __restrict__ wv, const HelZ* __restrict__ zw, const float* __restrict__ wtab,
               const float* __restrict__ ang, const float* __restrict__ zsrc, const float2* __restrict__ tab,
               float* __restrict__ out, const int nview, const int nzg, const double dvv) {
    __shared__ HelZ szw[R];
    __shared__ int sv[5];
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * NWY + threadIdx.y;
    const int zg = blockIdx.z % nzg, b = blockIdx.z / nzg;
    const int j0 = zg * R;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if (tid < R) {
        HelZ z;
        if (j0 + tid < g.D) z = zw[j0 + tid];
        else { z.vs = 1; z.ve = 0; z.bs = z.be = z.bc = z.pz = 0.0f; z.full = 1; z.pad = 0; }
        szw[tid] = z;
    }
    __syncthreads();
    if (tid == 0) {
        int lo = nview, hi = -1, allfull = 1, in_lo = 0, in_hi = nview - 1;
        for (int i = 0; i < R; ++i) {
            if (szw[i].vs <= szw[i].ve) { lo = min(lo, szw[i].vs); hi = max(hi, szw[i].ve); }
            allfull &= szw[i].full;
            in_lo = max(in_lo, szw[i].vs);
            in_hi = min(in_hi, szw[i].ve);
        }
        sv[0] = lo;
        sv[1] = hi;
        sv[2] = allfull;
        sv[3] = in_lo;  // views inside every slice's window: in_lo .. in_hi
        sv[4] = in_hi;
    }
    __syncthreads();
    // every slice's weight comes from the table: no exact fan angle needed
    // unless a test falls near an edge
    const bool allfull = sv[2] != 0;
    const int in_lo = sv[3], in_hi = sv[4];
    // slice i's centre z (for the approximate row test): pz_0 + i dz
    const float pz0 = szw[0].pz, dzf = (float)g.dz;
    const float row_off = 0.5f * (float)g.Nv - 0.5f;
    if (ix >= g.W || iy >= g.H || j0 >= g.D) return;
    const int Nu = g.Nu, Nv = g.Nv;
    const size_t vstride = (size_t)(Nv + 2) * Nu;
    const float px = hw_px(g, ix), py = hw_py(g, iy);
    const HelScanF s = *scan;
    float acc[R], valid[R];
#pragma unroll
    for (int i = 0; i < R; ++i) { acc[i] = 0.0f; valid[i] = 0.0f; }

    const float inv_dv = (float)(1.0 / g.dv);
    for (int v = sv[0]; v <= sv[1]; ++v) {
        const HelWView w = wv[v];
        const float rx = __fsub_rn(px, w.sx), ry = __fsub_rn(py, w.sy);
        const float rxy = sqrtf(__fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)));
        if (rxy <= 1.0e-6f) continue;
        const float xbv = w.cosv * px - w.sinv * py;
        const float ybv = w.sinv * px + w.cosv * py;
        bool col_in;
        float gamma = 0.0f;
        if (allfull) {
            col_in = hw_col_in_fast(g, w, px, py, xbv, ybv);
        } else {
            float rxe, rye, rxye;
            hw_ray(w, px, py, gamma, rxye, rxe, rye);
            col_in = hw_col_in(g, w, gamma);
        }
        const float tz = __fdividef(w.sdd, rxy);
        float wt[R];
        bool any = false;
        if (allfull && v >= in_lo && v <= in_hi) {
            // CTA-uniform: every slice tabulated and inside its window.  The
            // approximate row of slice i's centre ray is affine in i (the
            // slices' z are pz_0 + i dz up to rounding far inside the test's
            // band); the exact test runs near an edge, as in hw_row_in_fast.
            const float rk = tz * inv_dv;
            const float row0 = fmaf(fmaf(pz0 - w.szv, tz, w.szv - w.zs - (float)g.shv), inv_dv, row_off);
            const float drow = dzf * rk;
            const float top = (float)g.Nv - 0.5f;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const float wi = wtab[(size_t)(j0 + i) * nview + v];
                wt[i] = wi;
                if (wi != 0.0f) {
                    any = true;
                    if (col_in) {
                        const float row = fmaf((float)i, drow, row0);
                        bool in;
                        if (row > -0.5f + HW_BAND && row < top - HW_BAND) in = true;
                        else if (row < -0.5f - HW_BAND || row > top + HW_BAND) in = false;
                        else in = hw_row_in(g, w, rxy, szw[i].pz);
                        if (in) valid[i] += wi;
                    }
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const HelZ& z = szw[i];
                float wi = 0.0f;
                if (v >= z.vs && v <= z.ve)
                    wi = z.full ? wtab[(size_t)(j0 + i) * nview + v]
                                : hw_weight(o, g, px, py, z.pz, w.beta, gamma, w.szv, rxy, z.bc, z.bs, z.be, s.db,
                                            s.gmax, ang, zsrc, nview);
                wt[i] = wi;
                if (wi != 0.0f) {
                    any = true;
                    if (col_in && hw_row_in_fast(g, w, rxy, tz, inv_dv, z.pz)) valid[i] += wi;
                }
            }
        }
        if (!DD || !any) continue;
        const ViewHdr& h = vt.hdr[v];
        const HelView hv = vt.hel[v];
        const int keep = h.keep;
        int L, p;
        float xa, ya, xb, yb;
        if (h.use_x) {
            L = iy; p = ix;
            ya = yb = gf.yc0 - (float)L * gf.dy;
            xa = gf.x0 + (float)p * gf.dx;
            xb = xa + gf.dx;
        } else {
            L = ix; p = g.H - 1 - iy;
            xa = xb = gf.xc0 + (float)L * gf.dx;
            ya = gf.y0 + (float)p * gf.dy;
            yb = ya + gf.dy;
        }
        const double zs = (double)j0 + hv.z0dz;
        const double zoffh = hv.zoffh;
        const double q = fma(h.q1, (double)L, h.q0);
        const double mvdv = __drcp_rn(q * dvv);
        // column width SOD du over the squared source distance
        const float lf = __fdiv_rn(s.cwW, __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)));
        const float margin = 0.5f + XR_GUESS_ATAN_ERR * hv.inv_du;
        const float sf = (float)h.s, cf = (float)h.c;
        // one guess at the pixel centre and a bound on the footprint's
        // half-width: the pixel's edge segment on this line (half-length a,
        // at rxy from the source) spans at most a / (rxy - a) rad each side
        const float kc = col_guess_fast(gf, h, sf, cf, h.dcx, h.dcy, px, py, hv.inv_du);
        const float ha = 0.5f * (h.use_x ? gf.dx : gf.dy);
        const float hw = __fdividef(ha, fmaxf(rxy - ha, ha)) * hv.inv_du * 1.001f;
        const float kf0 = kc - hw, kf1 = kc + hw;
        const float lo = fmaxf(fminf(fminf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const float hi = fmaxf(fminf(fmaxf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const int ka = max(0, (int)floorf(lo - margin));
        const int kb = min(Nu - 1, (int)floorf(hi + margin));
        if (ka > kb) continue;
        const char* __restrict__ tvb = reinterpret_cast<const char*>(tab + ((size_t)b * nview + v) * vstride);
        const unsigned Nu8 = (unsigned)Nu * 8u;
        // Boundaries relative to the pixel: boundary ka in FP64, the next ones
        // by the columns' widths on this line in FP32; the run's row offset
        // and rows per voxel in FP64 at the first column, at the next ones
        // plus their FP32 changes (as in vox_prefix3d_kernel).
        const float4* __restrict__ cWR = vt.colWR + (size_t)v * Nu;
        const float Lf = (float)L;
        auto width = [&](int c) { const float4 wc = cWR[c]; return fmaf(wc.y, Lf, wc.x); };
        int k = ka;
        float pkl = (float)(fma(vt.bB[(size_t)v * (Nu + 1) + k], (double)L, vt.bA[(size_t)v * (Nu + 1) + k]) - (double)p);
        float pk1 = pkl + width(k);
        while (!(pk1 > 0.0f) && k < kb) {
            ++k;
            pkl = pk1;
            pk1 += width(k);
        }
        const float4 Wr = cWR[k];
        const double ibr = mvdv * ((double)Wr.z + (double)Wr.w);
        const double u0r = fma(zs, ibr, zoffh);
        const double tr0 = u0r + 6755399441055744.0;  // 1.5 * 2^52: rounds to an integer
        const int r0 = __double2loint(tr0);
        const float f0r = (float)(u0r - (tr0 - 6755399441055744.0));
        const float fibr = (float)ibr, mvdvf = (float)mvdv, zsf = (float)zs, r0f = (float)r0;
        // entry of local row n: tvb + ((r0 + 1 + n) Nu + col) 8
        //   = rb + col 8 + bits(n + 1.5 * 2^23) Nu8, bits read as unsigned
        const uintptr_t rb =
            reinterpret_cast<uintptr_t>(tvb) + (uintptr_t)((long long)(r0 + 1) * Nu8 - 0x4B400000ll * (long long)Nu8);
        // rows -1 .. Nv of the detector (table rows 0 .. Nv + 1)
        const float ulo = -1.0f - r0f, uhi = (float)Nv - 0.5f - r0f;
        for (;;) {
            const float wf = fminf(1.0f, pk1) - fmaxf(0.0f, pkl);
            if (wf > 0.0f) {
                const float4 Wk = cWR[k];
                const float dib = mvdvf * ((Wk.z - Wr.z) + (Wk.w - Wr.w));
                const float fib = fibr + dib;  // detector rows per voxel
                const float f0 = fmaf(zsf, dib, f0r);
                const float ub = f0 + r0f;
                // the guard keeps local row indices far below 2^22, where the
                // FP32 round-to-nearest by 1.5 * 2^23 below is exact
                if (fib < 4096.0f && ub < (float)Nv - 0.5f && fmaf((float)R, fib, ub) > -0.5f) {
                    const int col = keep ? k : Nu - 1 - k;
                    const char* cb = reinterpret_cast<const char*>(rb + (uintptr_t)col * 8u);
                    const float wk = __fdividef(wf * lf, fib);
                    float gprev = 0.0f;
#pragma unroll
                    for (int i = 0; i <= R; ++i) {
                        const float uc = fminf(fmaxf(fmaf((float)i, fib, f0), ulo), uhi);
                        const float tr = uc + 12582912.0f;  // round to nearest integer (FMA pipe)
                        const float nf = tr - 12582912.0f;
#ifdef XR_DEBUG_BOUNDS
                        const long long t = XR_BOUND((long long)r0 + 1 + (__float_as_int(tr) - 0x4B400000), 0, Nv + 1);
                        const float2 e = __ldg(reinterpret_cast<const float2*>(tvb) + (size_t)t * Nu + XR_BOUND(col, 0, Nu - 1));
#else
                        const float2 e = __ldg(reinterpret_cast<const float2*>(
                            cb + (size_t)(unsigned)__float_as_int(tr) * Nu8));
#endif
                        const float gi = fmaf(uc - nf, e.y, e.x);
                        if (i > 0) acc[i - 1] = fmaf(wk * wt[i - 1], gi - gprev, acc[i - 1]);
                        gprev = gi;
                    }
                }
            }
            if (++k > kb) break;
            pkl = pk1;
            if (pkl >= 1.0f) break;
            pk1 += width(k);
        }
    }
    const float ideal_db = (fabsf(s.db) > 1.0e-8f) ? __fdiv_rn(XR_PI_F, fabsf(s.db)) : -1.0f;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = j0 + i;
        if (j < g.D) {
            const size_t oi = ((size_t)j * g.H + iy) * g.W + ix;
            const float ideal = ideal_db >= 0.0f ? ideal_db : valid[i];
            const float sc = fminf(32.0f, fmaxf(0.03125f, __fdiv_rn(ideal, fmaxf(valid[i], 1.0e-6f))));
            if (DD) out[(size_t)b * g.D * g.H * g.W + oi] = acc[i] * sc;
            else if (b == 0) out[oi] = sc;
        }
    }
}

// -------------------------------------------------------------------- Bw^T

// img_s = img * scale (per voxel, every batch element).
__global__ void hel_prescale_kernel(const float* __restrict__ img, const float* __restrict__ scale,
                                    float* __restrict__ out, const size_t nvox, const size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = img[i] * scale[i % nvox];
}

// Cell gather of the weighted backprojection's transpose: thread = (view,
// detector column in traversal order, run of R rows), as cell_gather3d_kernel;
// every voxel of a column's footprint is weighted by its own redundancy
// weight (its slice's window, the pixel's fan angle) and read from the
// normalised image img_s.
//   ACCUM: add to `sino` the slices whose weights are not tabulated (the TMA
//          cell gather wrote the others); without it, every slice
template <int R, bool ACCUM>
__global__ void __launch_bounds__(256)
hel_wbpt_kernel(const Geom g, const ViewTables vt, const HelOpts o, const HelScanF* __restrict__ scan,
                const HelWView* __restrict__ wv, const HelZ* __restrict__ zw, const float* __restrict__ wtab,
                const float* __restrict__ ang,
                const float* __restrict__ zsrc, const float* __restrict__ img_s, const float* __restrict__ img_sT,
                float* __restrict__ sino, const int nview, const int view0, const double dvv) {
    // every slice tabulated: the weight of voxel j is wtab[j][v], with no
    // fan angle and no window test
    int full_here = 1;
    for (int i = threadIdx.y * 32 + threadIdx.x; i < g.D; i += blockDim.x * blockDim.y) full_here &= zw[i].full;
    const bool allfull = __syncthreads_and(full_here) != 0;
    if (ACCUM && allfull) return;  // nothing left to add
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int r0 = (blockIdx.y * blockDim.y + threadIdx.y) * R;
    const int vb = blockIdx.z + view0;
    const int v = vb % nview, b = vb / nview;
    const int Nu = g.Nu;
    if (k >= Nu || r0 >= g.Nv) return;
    const ViewHdr h = vt.hdr[v];
    const HelView hv = vt.hel[v];
    const HelWView w = wv[v];
    const HelScanF s = *scan;
    const float* __restrict__ wcol = wtab + v;  // wcol[j * nview] = weight of slice j
    const size_t ob = (size_t)v * (Nu + 1) + k;
    const double bA0 = vt.bA[ob], bB0 = vt.bB[ob], bA1 = vt.bA[ob + 1], bB1 = vt.bB[ob + 1];
    const double Qk = vt.colQ[(size_t)v * Nu + k];
    const int nlines = h.nlines, npix = h.npix;
    const size_t plane = (size_t)g.H * g.W;
    // lines of x-axis views are image rows; those of y-axis views are image
    // columns, read from the flipped transpose so that a warp's lanes (the
    // CTA's detector columns) stay on neighbouring addresses
    const float* __restrict__ vol = (h.use_x ? img_s : img_sT) + (size_t)b * g.D * plane;
    const int lpitch = h.use_x ? g.W : g.H;
    const double zr0 = hv.zd0 + r0 * dvv;
    float acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = 0.0f;

    for (int L = 0; L < nlines; ++L) {
        const double pk = fma(bB0, (double)L, bA0);
        const double pk1 = fma(bB1, (double)L, bA1);
        const int pa = max((int)floor(pk), 0);
        const int pb = min((int)ceil(pk1) - 1, npix - 1);
        if (pa > pb) continue;
        const double q = fma(h.q1, (double)L, h.q0);
        const double gq = Qk * q;
        const double t0 = fma(gq, zr0, -hv.z0dz);
        const double bt = gq * dvv;
        if (!(bt > 1.0e-4 && bt < 1.0e4)) continue;  // bounds every merge loop
        if (t0 + R * bt <= 0.0 || t0 >= (double)g.D) continue;
        const double jf = floor(t0);
        const int j0 = (int)jf;
        const float f = (float)(t0 - jf);
        const float bf = (float)bt;
        for (int p = pa; p <= pb; ++p) {
            const float wxy = (float)(fmin((double)p + 1.0, pk1) - fmax((double)p, pk));
            if (!(wxy > 0.0f)) continue;
            int ix, iy;
            if (h.use_x) { ix = p; iy = L; } else { ix = L; iy = g.H - 1 - p; }
            const float px = hw_px(g, ix), py = hw_py(g, iy);
            const float rx = __fsub_rn(px, w.sx), ry = __fsub_rn(py, w.sy);
            const float r2 = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
            const float rxy = sqrtf(r2);
            if (rxy <= 1.0e-6f) continue;
            float gamma = 0.0f;
            if (!allfull) {
                float rxe, rye, rxye;
                hw_ray(w, px, py, gamma, rxye, rxe, rye);
            }
            const float lf = wxy * __fdividef(s.cwW, r2);
            const float* __restrict__ col = vol + (size_t)L * lpitch + p;
            // value of voxel j of this column: weight x normalised image
            auto value = [&](int j) -> float {
                if ((unsigned)j >= (unsigned)g.D) return 0.0f;
                float wt;
                if (allfull) {
                    wt = __ldg(wcol + (size_t)j * nview);
                } else {
                    const HelZ z = zw[j];
                    if (v < z.vs || v > z.ve || (ACCUM && z.full)) return 0.0f;
                    wt = z.full ? __ldg(wcol + (size_t)j * nview)
                                : hw_weight(o, g, px, py, z.pz, w.beta, gamma, w.szv, rxy, z.bc, z.bs, z.be, s.db,
                                            s.gmax, ang, zsrc, nview);
                }
                return wt == 0.0f ? 0.0f : wt * __ldg(col + (size_t)j * plane);
            };
            int j = j0;
            float vj = value(j), pos = f, jn = 1.0f;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const float top = fmaf(bf, (float)(i + 1), f);
                float a = 0.0f;
                while (jn < top) {
                    a = fmaf(jn - pos, vj, a);
                    pos = jn;
                    ++j;
                    jn += 1.0f;
                    vj = value(j);
                }
                if (top > pos) { a = fmaf(top - pos, vj, a); pos = top; }
                acc[i] = fmaf(lf, a, acc[i]);
            }
        }
    }
    const int colo = h.keep ? k : Nu - 1 - k;
    float* out = sino + (((size_t)b * nview + v) * g.Nv) * Nu + colo;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int r = r0 + i;
        if (r < g.Nv) {
            if (ACCUM) out[(size_t)r * Nu] += acc[i];
            else out[(size_t)r * Nu] = acc[i];
        }
    }
}

}  // namespace xr
