// Voxel gather (B, Bw, A^T) through per-view row prefix tables.
//
// The z part of the DD backprojection of one (voxel column, detector column)
// pair is the overlap integral of the detector column y[r] (rows mapped to
// voxel z units at t_r = T0 + r*bt) with each voxel [j, j+1]:
//     Z(j) = bt * (G(u(j+1)) - G(u(j))),   u(z) = (z - T0) / bt,
//     G(u) = P[floor u] + (u - floor u) * y[floor u],  P[r] = sum_{r'<r} y[r'],
// the same sum the reference forms by merging row and voxel boundaries
// (include/cpu3d_common.h:48-202, backward3d_flat.cu:7-128), written as a
// difference of a piecewise-linear primitive.  Every voxel boundary costs one
// table lookup, independent of the data, so a warp never diverges on the
// number of rows a voxel overlaps.
//
// Table layout (one per batch element and view), float2 {C, y} indexed
// [row t = r + 1][physical column], rows t = 0 .. Nv + 1:
//     t = 0      : {P[0], 0}                (everything below row 0)
//     t = r + 1  : {P[r] + y[r] / 2, y[r]}  (primitive at the row's middle)
//     t = Nv + 1 : {P[Nv], 0}               (everything above the last row)
// so that G(u) = C[n] + (u - 1/2 - n) * y[n] for any n with |u - 1/2 - n| <= 1/2:
// the row index may be taken as round-to-nearest(u - 1/2), which an FP32 add
// of 1.5 * 2^23 yields on the FMA pipe (ties pick either neighbour; both give
// the same G).  Clamping u - 1/2 to [-1, Nv - 1/2] makes G exact outside the
// detector.  P is summed in FP64 and stored relative to the middle row
// (P[Nv/2] = 0), which halves the magnitude the FP32 differences cancel
// against.
#pragma once

#include "xr_kernels.cuh"

namespace xr {

// One thread per (batch element x view, physical column).  MODE OP_AT with a
// cone geometry folds the projection's cell scale s_A(k, r) into y, as
// prescale_at3d_kernel does.
template <typename TI, bool PRESCALE, bool HEL = false>
__global__ void __launch_bounds__(128)
row_prefix3d_kernel(const Geom g, const ViewTables vt, const TI* __restrict__ in, float2* __restrict__ tab,
                    const int nview, const int nbv, const double zd0_p, const double dvv) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int Nu = g.Nu, Nv = g.Nv;
    if (c >= Nu) return;
    for (int bv = blockIdx.y; bv < nbv; bv += gridDim.y) {
        const int v = bv % nview;
        const TI* __restrict__ src = in + (size_t)bv * Nv * Nu + c;
        float2* __restrict__ dst = tab + (size_t)bv * (Nv + 2) * Nu + c;
        float E = 1.0f, F = 0.0f, M = 0.0f;
        double zd0 = zd0_p;
        float zsrc = 0.0f;
        if (PRESCALE) {
            const int k = vt.hdr[v].keep ? c : Nu - 1 - c;
            const size_t oc = (size_t)v * Nu + k;
            E = vt.colE[oc]; F = vt.colF[oc]; M = vt.colM[oc];
            if (HEL) { zd0 = vt.hel[v].zd0; zsrc = vt.hel[v].zsrc; }
        }
        auto value = [&](int r) -> float {
            const float y = ld(src + (size_t)r * Nu);
            if (!PRESCALE) return y;
            float zc = (float)(zd0 + (r + 0.5) * dvv) * M;
            if (HEL) zc += zsrc;  // helical: the row's absolute z
            return y * E * sqrtf(F + zc * zc);
        };
        double half = 0.0;
        for (int r = 0; r < Nv / 2; ++r) half += (double)value(r);
        double run = -half;
        dst[0] = make_float2((float)run, 0.0f);
        for (int r = 0; r < Nv; ++r) {
            const float y = value(r);
            dst[(size_t)(r + 1) * Nu] = make_float2((float)(run + 0.5 * (double)y), y);
            run += (double)y;
        }
        dst[(size_t)(Nv + 1) * Nu] = make_float2((float)run, 0.0f);
    }
}

// FP32 detector-column guess for a point (traversal order, fractional
// boundary index).  Only used to bracket the columns a pixel overlaps; the
// overlaps themselves come from the FP64 boundary tables.  (dcx, dcy) is the
// arc detector's central direction for this view.
__device__ __forceinline__ float col_guess_fast(const GeomF& gf, const ViewHdr& h, float s, float c, float dcx,
                                                float dcy, float x, float y, float inv_du) {
    float sg;
    if (gf.type == GEO_FLAT) {
        const float R = gf.sod;
        const float u = __fdividef(R * (x * c + y * s), R + x * s - y * c);
        sg = (u * gf.inv_uscale - gf.shu) * inv_du;
    } else if (gf.type == GEO_ARC) {
        const float ex = x - (float)h.sx, ey = y - (float)h.sy;
        sg = guess_atan2f(dcx * ey - dcy * ex, dcx * ex + dcy * ey) * inv_du;
    } else {
        sg = (x * c + y * s - gf.shu) * inv_du;
    }
    return h.keep ? sg + 0.5f * gf.Nu : 0.5f * gf.Nu - sg;
}

// Voxel gather through the prefix tables.  CTA = 32 x NWY pixels of the image
// plane (lane = x, warp = y) times one run of R voxels along z per thread, so
// the warps of a CTA read overlapping parts of each view's table; the view
// loop is inside the kernel, so each voxel is written once and no atomics are
// needed.
//   MODE OP_B  : T_vox weight cw / ((X_hi - X_lo) Mv dz) in pixel units
//   MODE OP_BW : OP_B times the FBP distance weight of the voxel centre
//   MODE OP_AT : adjoint of the projection (cone: the table holds the
//                pre-scaled sinogram; the line factor dpix dz / q^2)
#ifndef XR_PFX_MINB
#define XR_PFX_MINB 4
#endif
//   HEL        : helical scan; the view's z placement, column width and
//                angular column pitch come from vt.hel
//   CHAIN      : circular arc detector, B / Bw: the pixel's columns are
//                walked with the reference's chained float32 angles
//                (ArcChain, vt.arc)
template <typename TO, int R, int NWY, int MODE, bool HEL = false, bool CHAIN = false>
__global__ void __launch_bounds__(32 * NWY, XR_PFX_MINB)
vox_prefix3d_kernel(const Geom g, const GeomF gf, const ViewTables vt, const float2* __restrict__ tab,
                    TO* __restrict__ vol, const int nview, const int nzg, const double z0dz, const double zd0,
                    const double dvv, const float cw, const float atconst, const float oscale) {
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * NWY + threadIdx.y;
    const int zg = blockIdx.z % nzg, b = blockIdx.z / nzg;
    const int j0 = zg * R;
    if (ix >= g.W || iy >= g.H || j0 >= g.D) return;
    const int Nu = g.Nu, Nv = g.Nv;
    const unsigned Nu8 = (unsigned)Nu * 8u;
    const size_t vstride = (size_t)(Nv + 2) * Nu;
    const float2* __restrict__ tb = tab + (size_t)b * nview * vstride;
    double zs = (double)j0 + z0dz;  // run bottom, in voxel units from z = 0
    double zoffh = -zd0 / dvv - 0.5;  // u0 = zs * (rows per voxel) + zoffh
    const float dpdz = (float)g.dz;
    // column bracket margin: half a column, plus the arc guess's angle error
    float inv_du = gf.inv_du;
    float margin = 0.5f + (g.type == GEO_ARC ? XR_GUESS_ATAN_ERR * inv_du : 0.0f);
    // world z range of the run (helical view skipping)
    const float zrun_lo = (float)((-0.5 * g.D + j0) * g.dz + g.shz);
    const float zrun_hi = (float)((-0.5 * g.D + min(j0 + R, g.D)) * g.dz + g.shz);
    float acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = 0.0f;

    for (int v = 0; v < nview; ++v) {
        const ViewHdr& h = vt.hdr[v];
        const int keep = h.keep;
        float cwv = cw;
        if (HEL) {
            const HelView hv = vt.hel[v];
            // CTA-uniform: the whole z run lies outside what this view reaches
            if (zrun_hi < hv.zlo || zrun_lo > hv.zhi) continue;
            zs = (double)j0 + hv.z0dz;
            zoffh = hv.zoffh;
            cwv = hv.cw;
            inv_du = hv.inv_du;
            margin = 0.5f + XR_GUESS_ATAN_ERR * inv_du;
        }
        int L, p;
        float xa, ya, xb, yb, px, py;
        if (h.use_x) {
            L = iy; p = ix;
            ya = yb = py = gf.yc0 - (float)L * gf.dy;
            xa = gf.x0 + (float)p * gf.dx;
            xb = xa + gf.dx;
            px = xa + 0.5f * gf.dx;
        } else {
            L = ix; p = g.H - 1 - iy;
            xa = xb = px = gf.xc0 + (float)L * gf.dx;
            ya = gf.y0 + (float)p * gf.dy;
            yb = ya + gf.dy;
            py = ya + 0.5f * gf.dy;
        }
        const double q = fma(h.q1, (double)L, h.q0);
        const double mvdv = __drcp_rn(q * dvv);  // rows per voxel = mvdv * colR[k]
        float lf;
        if (MODE == OP_AT) {
            if (g.type == GEO_PARALLEL) lf = atconst;
            else { const float qf = (float)q; lf = (float)h.dpix * dpdz / (qf * qf); }
        } else {
            lf = cwv;
            if (MODE == OP_BW) lf *= fbp_weight(g, h, px, py);
        }
        lf *= oscale;
        const float sf = (float)h.s, cf = (float)h.c;
        const float dcx = h.dcx, dcy = h.dcy;
        float kf0, kf1;
        if (CHAIN) {  // arc detector (the other instantiations keep two guesses: fewer live registers)
            // one guess at the pixel centre and a bound on the footprint's
            // half-width: the pixel's edge segment on this line (half-length
            // a, distance r from the source) spans at most a / (r - a) rad
            // each side of the centre
            const float kc = col_guess_fast(gf, h, sf, cf, dcx, dcy, px, py, inv_du);
            const float ex = px - (float)h.sx, ey = py - (float)h.sy;
            const float a = 0.5f * (h.use_x ? gf.dx : gf.dy);
            const float r2 = fmaf(ex, ex, ey * ey);
            const float hw = __fdividef(a, fmaxf(r2 * rsqrtf(r2) - a, a)) * inv_du * 1.001f;
            kf0 = kc - hw;
            kf1 = kc + hw;
        } else {
            kf0 = col_guess_fast(gf, h, sf, cf, dcx, dcy, xa, ya, inv_du);
            kf1 = col_guess_fast(gf, h, sf, cf, dcx, dcy, xb, yb, inv_du);
        }
        const float lo = fmaxf(fminf(fminf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const float hi = fmaxf(fminf(fmaxf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const int ka = max(0, (int)floorf(lo - margin));
        const int kb = min(Nu - 1, (int)floorf(hi + margin));
        if (ka > kb) continue;
        const char* __restrict__ tvb = reinterpret_cast<const char*>(tb + (size_t)v * vstride);
        const float4* __restrict__ cWR = vt.colWR + (size_t)v * Nu;
        const float Lf = (float)L;
        // Boundaries relative to the pixel, in pixel units: boundary ka in
        // FP64, the next ones by adding the columns' widths on this line in
        // FP32 (pd: the direct boundary k + 1).  First column whose right
        // boundary lies right of the pixel's left edge:
        int k = ka;
        float pkl = (float)(fma(vt.bB[(size_t)v * (Nu + 1) + k], (double)L, vt.bA[(size_t)v * (Nu + 1) + k]) - (double)p);
        auto width = [&](int c) { const float4 w = cWR[c]; return fmaf(w.y, Lf, w.x); };
        float pd = pkl + width(k);
        while (!(pd > 0.0f) && k < kb) {
            ++k;
            pkl = pd;
            pd += width(k);
        }
        float pk1 = pd;
        ArcChain ch;
        float qd = 0.0f;
        const float4* __restrict__ ea = nullptr;
        if (CHAIN) {
            ea = vt.arc + 2 * (size_t)v * (Nu + 1);
            qd = __fdividef((float)q, h.use_x ? gf.dx : gf.dy);  // pixels per axis unit on this line (scales the chain's small offsets)
            ch.start(ea, k, keep, gf.du);
            float d = ch.next_linear(ea, k + 1);
            if (k + 1 == Nu) d = fminf(d, 0.0f);  // the detector's end
            pk1 = fmaf(d, qd, pd);
        }
        // The run's rows at column k: its bottom boundary minus half a row is
        // u0 = zs ib + zoffh, ib = mvdv colR[k] rows per voxel.  Evaluated in
        // FP64 at this first column (kr) and split into an integer row r0
        // and f0 = u0 - r0; at the others u0 - r0 = f0 + zs (ib - ib_kr) and
        // ib - ib_kr = mvdv (colR[k] - colR[kr]), both small, in FP32 (the
        // colR difference from the hi + lo pairs, hi - hi exact).
        const float4 Wr = cWR[k];
        const float2 Rr = make_float2(Wr.z, Wr.w);
        const double ibr = mvdv * ((double)Rr.x + (double)Rr.y);
        const double u0r = fma(zs, ibr, zoffh);
        const double tr0 = u0r + 6755399441055744.0;  // 1.5 * 2^52: rounds to an integer
        const int r0 = __double2loint(tr0);
        const float f0r = (float)(u0r - (tr0 - 6755399441055744.0));
        const float fibr = (float)ibr, mvdvf = (float)mvdv, zsf = (float)zs, r0f = (float)r0;
        // Address of the entry for local row n of column col:
        //   tvb + ((r0 + 1 + n) Nu + col) 8 = rb + col 8 + bits(n + 1.5 * 2^23) Nu8
        // with bits() read as unsigned: one wide multiply-add per lookup.
        const uintptr_t rb =
            reinterpret_cast<uintptr_t>(tvb) + (uintptr_t)((long long)(r0 + 1) * Nu8 - 0x4B400000ll * (long long)Nu8);
        // lanes now walk their overlapping columns in step, one per iteration
        for (;;) {
            const float wf = fminf(1.0f, pk1) - fmaxf(0.0f, pkl);
            do {
                if (!(wf > 0.0f)) break;
                const float4 Wk = cWR[k];
                const float dib = mvdvf * ((Wk.z - Rr.x) + (Wk.w - Rr.y));
                const float fib = fibr + dib;  // detector rows per voxel
                // keeps every local row index below 2^17, where the FP32
                // round-to-nearest below is exact (geometries this extreme
                // are far outside any scanner's)
                if (!(fib < 4096.0f)) break;
                const float f0 = fmaf(zsf, dib, f0r);
                const float ub = f0 + r0f;                 // the run's rows, detector coordinates
                const float ut = fmaf((float)R, fib, ub);
                if (ub >= (float)Nv - 0.5f || ut <= -0.5f) break;
                const int col = keep ? k : Nu - 1 - k;
                const char* cb = reinterpret_cast<const char*>(rb + (uintptr_t)col * 8u);
                // the table entry of a row rounded by the 1.5 * 2^23 add: local row
                // bits(tr) - bits(1.5 * 2^23), table row r0 + 1 + that
#ifdef XR_DEBUG_BOUNDS
                auto entry = [&](float tr) -> float2 {
                    const long long t = XR_BOUND((long long)r0 + 1 + (__float_as_int(tr) - 0x4B400000), 0, Nv + 1);
                    return __ldg(reinterpret_cast<const float2*>(tvb) + (size_t)t * Nu + XR_BOUND(col, 0, Nu - 1));
                };
#else
                auto entry = [&](float tr) -> float2 {
                    return __ldg(reinterpret_cast<const float2*>(cb + (size_t)(unsigned)__float_as_int(tr) * Nu8));
                };
#endif
                const float wk = __fdividef(wf * lf, fib);
                // rows the run reaches, inside [0, Nv - 1] in every active lane?
                const bool inside = (ub >= 0.0f) && (ut <= (float)(Nv - 1));
                float gprev = 0.0f;
                if (__all_sync(__activemask(), inside)) {
                    // boundaries in pairs: the index arithmetic on packed FP32x2
                    const float2 fib2 = make_float2(fib, fib), f02 = make_float2(f0, f0);
                    const float2 mg2 = make_float2(12582912.0f, 12582912.0f);  // 1.5 * 2^23
                    const float2 nmg2 = make_float2(-12582912.0f, -12582912.0f);
                    const float2 neg2 = make_float2(-1.0f, -1.0f);
#pragma unroll
                    for (int i = 0; i <= R; i += 2) {
                        if (i + 1 <= R) {
                            const float2 u2 = __ffma2_rn(make_float2((float)i, (float)(i + 1)), fib2, f02);
                            const float2 tr2 = __fadd2_rn(u2, mg2);   // round to nearest integer
                            const float2 nf2 = __fadd2_rn(tr2, nmg2);
                            const float2 fr2 = __ffma2_rn(nf2, neg2, u2);  // u - n
                            const float2 ea = entry(tr2.x);
                            const float2 eb = entry(tr2.y);
                            const float ga = fmaf(fr2.x, ea.y, ea.x);
                            const float gb = fmaf(fr2.y, eb.y, eb.x);
                            if (i > 0) acc[i - 1] = fmaf(wk, ga - gprev, acc[i - 1]);
                            acc[i] = fmaf(wk, gb - ga, acc[i]);
                            gprev = gb;
                        } else {
                            const float uc = fmaf((float)i, fib, f0);
                            const float tr = uc + 12582912.0f;
                            const float nf = tr - 12582912.0f;
                            const float2 e = entry(tr);
                            const float gi = fmaf(uc - nf, e.y, e.x);
                            acc[i - 1] = fmaf(wk, gi - gprev, acc[i - 1]);
                        }
                    }
                } else {
                    const float ulo = -1.0f - r0f, uhi = (float)Nv - 0.5f - r0f;
#pragma unroll
                    for (int i = 0; i <= R; ++i) {
                        const float uc = fminf(fmaxf(fmaf((float)i, fib, f0), ulo), uhi);
                        const float tr = uc + 12582912.0f;
                        const float nf = tr - 12582912.0f;
                        const float2 e = entry(tr);
                        const float gi = fmaf(uc - nf, e.y, e.x);
                        if (i > 0) acc[i - 1] = fmaf(wk, gi - gprev, acc[i - 1]);
                        gprev = gi;
                    }
                }
            } while (false);
            if (++k > kb) break;
            pkl = pk1;
            if (pkl >= 1.0f) break;  // column k starts right of the pixel
            pd += width(k);
            pk1 = pd;
            if (CHAIN) {
                float d = ch.next_linear(ea, k + 1);
                if (k + 1 == Nu) d = fminf(d, 0.0f);
                pk1 = fmaf(d, qd, pd);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = j0 + i;
        if (j < g.D) st(vol + (((size_t)b * g.D + j) * g.H + iy) * g.W + ix, acc[i]);
    }
}

}  // namespace xr
