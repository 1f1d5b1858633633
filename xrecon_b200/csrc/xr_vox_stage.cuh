// Voxel gather (B, Bw, A^T) with TMA-staged row-prefix tables.
//
// Flat, parallel and arc detectors (CHAIN: B and Bw on arc detectors, whose
// columns are walked with the reference's chained float32 angles, as in
// vox_prefix3d_kernel).  The arithmetic per (pixel, view, column) is
// that of vox_prefix3d_kernel (xr_vox_prefix.cuh), and so are the results
// when every view is staged; what changes is where the table lookups go.
//
// CTA = a PS_T x PS_T tile of the image plane times one run of R voxels along
// z per thread (one pixel per thread).  For every view, the CTA's lookups fall
// in a box of that view's table:
//   columns: the brackets of the tile's four corners (the column coordinate
//            is a projective, so monotone, function of the point along any
//            line: every pixel's bracket lies between the corners'), widened
//            by the brackets' half column and one column more;
//   rows:    the rows the z-run reaches at the extremes of the rows-per-voxel
//            factor colR / (q dvv) over those columns and the tile's lines
//            (colR is linear in the column on flat detectors and a sinusoid
//            of the column angle on arc ones, whose distance from its chord
//            over the box is at most amplitude * width^2 / 8; q is linear in
//            the line), one row of margin each side.
// One thread copies each view's box into a ring of PS_NS stages with a tiled
// TMA load, PS_NS views ahead of the consumers; the lookups are shared-memory
// loads with 32-bit addresses.  A global-memory lookup of the same table, even
// an L1 hit, takes several times as long, and it was most of the kernel's
// time.
//
// Every lookup stays inside its stage by construction, whatever the box:
// the consumers clamp their column brackets to the box's columns, take the
// clamp-free lookups only for runs whose rows lie inside the box, and clamp
// the other runs' rows into it.  (With a correct box none of these clamps
// binds except at the detector's own edges, where the plain kernel clamps
// too.)  A view whose box exceeds the stage is not staged: the CTA skips it
// and records that it did, and the FALLBACK instantiation, launched after
// it, adds the skipped views' contributions from the tables in global
// memory.
//
// Windows are evaluated PS_WCH views at a time, one view per thread, into a
// double-buffered table in shared memory.
#pragma once

#include "xr_vox_prefix.cuh"
#include "xr_tma.cuh"

namespace xr {

constexpr int PS_T = 16;    // tile edge, pixels
constexpr int PS_NS = 2;    // stages of the ring
constexpr int PS_WCH = 64;  // views per window chunk

// Test hook: every odd view is reported as not fitting its stage, so the
// fallback launch does half the work.
constexpr unsigned XR_HOOK_PFX_UNFIT = 4u;
// Test hook, read on the host: the prefix gathers use vox_prefix3d_kernel
// (no staging).
constexpr unsigned XR_HOOK_PFX_NOSTAGE = 8u;

// Bytes of one stage: BR rows of BC float2, rounded up to 128 bytes.
__host__ __device__ inline size_t pfx_stage_bytes(int BC, int BR) {
    return ((size_t)BC * BR * sizeof(float2) + 127) / 128 * 128;
}
// Dynamic shared memory of the staged kernel: window table, barriers, ring.
__host__ __device__ inline size_t pfx_stage_smem(int BC, int BR) {
    return 2 * PS_WCH * sizeof(int4) + 128 + PS_NS * pfx_stage_bytes(BC, BR);
}

// Box of view v for the CTA at tile (ix0, iy0) and z-run bottom zs:
//   {table column c0 (even, the TMA's 16-byte rule), table row r0,
//    first and last traversal column klo, khi}.
// klo > khi: nothing of the tile reaches the view (nothing to stage).
// c0 < 0: the box does not fit BC x BR (the view is left to the fallback).
// HEL: helical scan; the view's z placement and angular column pitch come
// from vt.hel (zs and zoffh are then the view's, from the run's first voxel
// j0), and a view whose z reach misses the run has nothing to stage.
// CHAIN: the consumers bracket a pixel by one guess at its centre and a
// bound on its footprint's half-width, a / (r - a) rad (a the half-length of
// the pixel's edge segment, r its distance from the source); the box widens
// by that bound at the least distance from the source to the tile, so that
// no bracket is clamped and every chain starts where the unstaged kernel's
// does.
template <bool HEL, bool CHAIN>
__device__ inline int4 pfx_window(const Geom& g, const GeomF& gf, const ViewTables& vt, const int v, const int ix0,
                                  const int iy0, const int j0, double zs, double zoffh, const double dvv, const int R,
                                  const int BC, const int BR) {
    const int4 unfit = make_int4(-1, 0, 0, 0), none = make_int4(0, 0, 1, 0);
    if ((*(volatile unsigned*)&g_test_hooks & XR_HOOK_PFX_UNFIT) && (v & 1)) return unfit;
    const ViewHdr& h = vt.hdr[v];
    float inv_du = gf.inv_du;
    double du = g.du;
    if (HEL) {
        const HelView& hv = vt.hel[v];
        const float zrun_lo = (float)((-0.5 * g.D + j0) * g.dz + g.shz);
        const float zrun_hi = (float)((-0.5 * g.D + min(j0 + R, g.D)) * g.dz + g.shz);
        if (zrun_hi < hv.zlo || zrun_lo > hv.zhi) return none;
        zs = (double)j0 + hv.z0dz;
        zoffh = hv.zoffh;
        inv_du = hv.inv_du;
        du = 1.0 / (double)hv.inv_du;
    }
    const int ixe = min(ix0 + PS_T, g.W) - 1, iye = min(iy0 + PS_T, g.H) - 1;
    // the tile's points as the consumers place them (segment ends of each
    // pixel on its line) and its first and last line
    float xl, xr, yl, yh;
    int L0, L1;
    if (h.use_x) {
        L0 = iy0; L1 = iye;
        xl = gf.x0 + (float)ix0 * gf.dx;
        xr = gf.x0 + (float)(ixe + 1) * gf.dx;
        yh = gf.yc0 - (float)L0 * gf.dy;
        yl = gf.yc0 - (float)L1 * gf.dy;
    } else {
        L0 = ix0; L1 = ixe;
        xl = gf.xc0 + (float)L0 * gf.dx;
        xr = gf.xc0 + (float)L1 * gf.dx;
        yl = gf.y0 + (float)(g.H - 1 - iye) * gf.dy;
        yh = gf.y0 + (float)(g.H - iy0) * gf.dy;
    }
    const float sf = (float)h.s, cf = (float)h.c;
    float gmin = 3.0e38f, gmax = -3.0e38f;
    auto corner = [&](float x, float y) {
        const float k = col_guess_fast(gf, h, sf, cf, h.dcx, h.dcy, x, y, inv_du);
        gmin = fminf(gmin, k);
        gmax = fmaxf(gmax, k);
    };
    corner(xl, yl); corner(xl, yh); corner(xr, yl); corner(xr, yh);
    const float lo = fmaxf(fminf(gmin, (float)g.Nu + 2.0f), -2.0f);
    const float hi = fmaxf(fminf(gmax, (float)g.Nu + 2.0f), -2.0f);
    // the consumers' half column and guess error, the corners' guess error, one column
    float wm = 1.5f + (HEL || g.type == GEO_ARC ? 2.0f * XR_GUESS_ATAN_ERR * inv_du : 0.0f);
    if (CHAIN) {
        // least distance from the source to the tile (the pixel centres lie inside it)
        const float ddx = fmaxf(fmaxf(xl - (float)h.sx, (float)h.sx - xr), 0.0f);
        const float ddy = fmaxf(fmaxf(yl - (float)h.sy, (float)h.sy - yh), 0.0f);
        const float rlo = sqrtf(ddx * ddx + ddy * ddy) * 0.9999f;
        const float a = 0.5f * (h.use_x ? gf.dx : gf.dy);
        wm += a / fmaxf(rlo - a, a) * inv_du * 1.002f;
    }
    const int kw0 = max(0, (int)floorf(lo - wm)), kw1 = min(g.Nu - 1, (int)floorf(hi + wm));
    if (kw0 > kw1) return none;
    // rows per voxel ib = colR / (q dvv) at its extremes over the box
    const double d0 = fma(h.q1, (double)L0, h.q0) * dvv, d1 = fma(h.q1, (double)L1, h.q0) * dvv;
    double Ra = vt.colR[(size_t)v * g.Nu + kw0], Rb = vt.colR[(size_t)v * g.Nu + kw1];
    double slack = 0.0;
    if (g.type == GEO_ARC) {
        // colR = dz (1 -/+ sdd trig(angle) / sperp): amplitude dz sdd / |sperp|
        const double wd = (double)(kw1 - kw0 + 1) * du;
        slack = 1.01 * g.dz * g.sdd / fabs(h.sperp) * wd * wd / 8.0 + 1e-12;
    }
    const double Rlo = fmin(Ra, Rb) - slack, Rhi = fmax(Ra, Rb) + slack;
    if (!(d0 > 0.0 && d1 > 0.0 && Rlo > 0.0)) return unfit;
    const double ibmin = Rlo / fmax(d0, d1), ibmax = Rhi / fmin(d0, d1);
    const double zt = zs + (double)R;
    const double ulo = zoffh + fmin(zs * ibmin, zs * ibmax), uhi = zoffh + fmax(zt * ibmin, zt * ibmax);
    // table row of detector coordinate d: 1 + round(d); one row of margin
    if (!(ulo <= uhi) || ulo > (double)g.Nv + 2.0 || uhi < -3.0) return none;
    const int rlo = max(0, (int)floor(fmax(ulo, -4.0))), rhi = min(g.Nv + 1, (int)ceil(fmin(uhi, (double)g.Nv + 4.0)) + 2);
    if (rlo > rhi) return none;
    const int c0 = (h.keep ? kw0 : g.Nu - 1 - kw1) & ~1;
    const int c1 = h.keep ? kw1 : g.Nu - 1 - kw0;
    if (c1 - c0 + 1 > BC || rhi - rlo + 1 > BR) return unfit;
    return make_int4(c0, rlo, kw0, kw1);
}

// 3D tiled TMA load of one box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

#ifndef XR_PFXS_MINB
#define XR_PFXS_MINB 4
#endif

// map: the tables as {Nu columns, Nv + 2 rows, batch x views} of 8-byte
// elements, box {BC, BR, 1}.  unfit[cta]: set by the staged launch when it
// skipped a view; the FALLBACK launch does only those CTAs' skipped views,
// adding to what the staged launch stored.
template <typename TO, int R, int MODE, bool FALLBACK, bool HEL = false, bool CHAIN = false>
__global__ void __launch_bounds__(PS_T * PS_T, XR_PFXS_MINB)
vox_stage3d_kernel(const Geom g, const GeomF gf, const ViewTables vt, const __grid_constant__ CUtensorMap map,
                   const float2* __restrict__ tab, TO* __restrict__ vol, int* __restrict__ unfit, const int nview,
                   const int nzg, const double z0dz, const double zd0, const double dvv, const float cw,
                   const float atconst, const float oscale, const int BC, const int BR) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    int4* wins = reinterpret_cast<int4*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * PS_WCH * sizeof(int4));
    unsigned char* stages = smem_raw + 2 * PS_WCH * sizeof(int4) + 128;
    const size_t stage_bytes = pfx_stage_bytes(BC, BR);

    const int tid = threadIdx.x;
    const int ix0 = blockIdx.x * PS_T, iy0 = blockIdx.y * PS_T;
    const int ix = ix0 + (tid % PS_T), iy = iy0 + (tid / PS_T);
    const int zg = blockIdx.z % nzg, b = blockIdx.z / nzg;
    const int j0 = zg * R;
    const bool active = ix < g.W && iy < g.H && j0 < g.D;
    const unsigned cta = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (FALLBACK && unfit[cta] == 0) return;  // CTA-uniform

    const int Nu = g.Nu, Nv = g.Nv;
    const unsigned Nu8 = (unsigned)Nu * 8u;
    const size_t vstride = (size_t)(Nv + 2) * Nu;
    const float2* __restrict__ tb = tab + (size_t)b * nview * vstride;
    const double zs0 = (double)j0 + z0dz;  // run bottom, in voxel units from z = 0
    const double zoffh0 = -zd0 / dvv - 0.5;  // u0 = zs * (rows per voxel) + zoffh
    const float dpdz = (float)g.dz;


    __shared__ int s_abort, s_unfit;
    volatile int* abort = &s_abort;
    if (tid == 0) {
        if (!FALLBACK) {
            for (int i = 0; i < PS_NS; ++i) mbar_init(&bar[i], 1);
            fence_barrier_init();
        }
        s_abort = 0;
        s_unfit = 0;
    }
    auto windows = [&](int vbase) {
        if (tid < PS_WCH && vbase + tid < nview) {
            const int4 w = pfx_window<HEL, CHAIN>(g, gf, vt, vbase + tid, ix0, iy0, j0, zs0, zoffh0, dvv, R, BC, BR);
            wins[((vbase / PS_WCH) & 1) * PS_WCH + tid] = w;
            if (w.x < 0) s_unfit = 1;
        }
    };
    auto window_of = [&](int v) { return wins[((v / PS_WCH) & 1) * PS_WCH + v % PS_WCH]; };
    windows(0);
    __syncthreads();

    // test hook: arm the barrier for a box but issue no copy
    const bool stall = (*(volatile unsigned*)&g_test_hooks & XR_HOOK_TMA_STALL) != 0;
    const unsigned box_bytes = (unsigned)((size_t)BC * BR * sizeof(float2));
    auto issue = [&](int v) {
        const int4 w = window_of(v);
        uint64_t* br = &bar[v % PS_NS];
        if (w.x >= 0 && w.z <= w.w) {
            mbar_arrive_expect_tx(br, box_bytes);
            if (!stall) tma_load_3d(stages + (size_t)(v % PS_NS) * stage_bytes, &map, w.x, w.y, b * nview + v, br);
        } else {
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(br)) : "memory");
        }
    };
    int last = -1;  // last view issued (issuing thread)
    if (!FALLBACK && tid == 0)
        for (int v = 0; v < min(PS_NS, nview); ++v) issue(v), last = v;

    float acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = 0.0f;
    if (FALLBACK && active) {
#pragma unroll
        for (int i = 0; i < R; ++i)
            if (j0 + i < g.D) acc[i] = ld(vol + (((size_t)b * g.D + j0 + i) * g.H + iy) * g.W + ix);
    }

    for (int v = 0; v < nview; ++v) {
        const int4 w = window_of(v);
        const bool mine = FALLBACK ? (w.x < 0) : (w.x >= 0 && w.z <= w.w);
        if (!FALLBACK && mine) mbar_wait_bounded(&bar[v % PS_NS], (unsigned)((v / PS_NS) & 1), abort);
        if (mine && active && !(!FALLBACK && *abort)) do {
            const ViewHdr& h = vt.hdr[v];
            const int keep = h.keep;
            // the view's z placement, column width and angular pitch
            // (helical), and the column bracket margin: half a column, plus
            // the arc guess's angle error
            double zs = zs0, zoffh = zoffh0;
            float cwv = cw, inv_du = gf.inv_du;
            if (HEL) {
                const HelView& hv = vt.hel[v];
                zs = (double)j0 + hv.z0dz;
                zoffh = hv.zoffh;
                cwv = hv.cw;
                inv_du = hv.inv_du;
            }
            const float margin = 0.5f + (HEL || g.type == GEO_ARC ? XR_GUESS_ATAN_ERR * inv_du : 0.0f);
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
            float kf0, kf1;
            if (CHAIN) {
                // one guess at the pixel centre and the footprint's half-width bound
                const float kc = col_guess_fast(gf, h, sf, cf, h.dcx, h.dcy, px, py, inv_du);
                const float ex = px - (float)h.sx, ey = py - (float)h.sy;
                const float a = 0.5f * (h.use_x ? gf.dx : gf.dy);
                const float r2 = fmaf(ex, ex, ey * ey);
                const float hw = __fdividef(a, fmaxf(r2 * rsqrtf(r2) - a, a)) * inv_du * 1.001f;
                kf0 = kc - hw;
                kf1 = kc + hw;
            } else {
                kf0 = col_guess_fast(gf, h, sf, cf, h.dcx, h.dcy, xa, ya, inv_du);
                kf1 = col_guess_fast(gf, h, sf, cf, h.dcx, h.dcy, xb, yb, inv_du);
            }
            const float lo = fmaxf(fminf(fminf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
            const float hi = fmaxf(fminf(fmaxf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
            // staged views: the bracket within the box's columns; the rows of
            // the clamp-free lookups and the clamps within its rows
            const int klo = FALLBACK ? 0 : w.z, khi = FALLBACK ? Nu - 1 : w.w;
            const int ka = max(klo, (int)floorf(lo - margin));
            const int kb = min(khi, (int)floorf(hi + margin));
            if (ka > kb) break;
            const float in_lo = FALLBACK ? 0.0f : (float)max(0, w.y - 1);
            const float in_hi = FALLBACK ? (float)(Nv - 1) : fminf((float)(Nv - 1), (float)(w.y + BR - 2));
            const float lo_d = FALLBACK ? -1.0f : (float)max(-1, w.y - 1);
            // (hi_d >= lo_d: a clamp into the box never lands below it)
            const float hi_d = FALLBACK ? (float)Nv - 0.5f : fmaxf(lo_d, fminf((float)Nv - 0.5f, (float)(w.y + BR - 2)));
            const float4* __restrict__ cWR = vt.colWR + (size_t)v * Nu;
            const float Lf = (float)L;
            int k = ka;
            float pkl = (float)(fma(vt.bB[(size_t)v * (Nu + 1) + k], (double)L, vt.bA[(size_t)v * (Nu + 1) + k]) - (double)p);
            auto width = [&](int c) { const float4 wc = cWR[c]; return fmaf(wc.y, Lf, wc.x); };
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
                qd = __fdividef((float)q, h.use_x ? gf.dx : gf.dy);  // pixels per axis unit on this line
                ch.start(ea, k, keep, gf.du);
                float d = ch.next_linear(ea, k + 1);
                if (k + 1 == Nu) d = fminf(d, 0.0f);  // the detector's end
                pk1 = fmaf(d, qd, pd);
            }
            const float4 Wr = cWR[k];
            const float2 Rr = make_float2(Wr.z, Wr.w);
            const double ibr = mvdv * ((double)Rr.x + (double)Rr.y);
            const double u0r = fma(zs, ibr, zoffh);
            const double tr0 = u0r + 6755399441055744.0;  // 1.5 * 2^52: rounds to an integer
            const int r0 = __double2loint(tr0);
            const float f0r = (float)(u0r - (tr0 - 6755399441055744.0));
            const float fibr = (float)ibr, mvdvf = (float)mvdv, zsf = (float)zs, r0f = (float)r0;
            // Entry of local row n of table column col, addressed with the
            // rounded value's bits as in the plain kernel: staged, a 32-bit
            // shared-memory offset relative to the box (modular arithmetic;
            // the sum is the entry's offset); fallback, the global table.
            const unsigned P = FALLBACK ? Nu8 : (unsigned)BC * 8u;
            const unsigned rb32 = (unsigned)(r0 + 1 - (FALLBACK ? 0 : w.y)) * P - 0x4B400000u * P;
            const unsigned char* sbase = stages + (size_t)(v % PS_NS) * stage_bytes;
            const char* __restrict__ tvb = reinterpret_cast<const char*>(tb + (size_t)v * vstride);
            for (;;) {
                const float wf = fminf(1.0f, pk1) - fmaxf(0.0f, pkl);
                do {
                    if (!(wf > 0.0f)) break;
                    const float4 Wk = cWR[k];
                    const float dib = mvdvf * ((Wk.z - Rr.x) + (Wk.w - Rr.y));
                    const float fib = fibr + dib;  // detector rows per voxel
                    if (!(fib < 4096.0f)) break;
                    const float f0 = fmaf(zsf, dib, f0r);
                    const float ub = f0 + r0f;                 // the run's rows, detector coordinates
                    const float ut = fmaf((float)R, fib, ub);
                    if (ub >= (float)Nv - 0.5f || ut <= -0.5f) break;
                    const int col = keep ? k : Nu - 1 - k;
                    const unsigned cb = rb32 + (unsigned)(col - (FALLBACK ? 0 : w.x)) * 8u;
                    auto entry = [&](float tr) -> float2 {
                        const unsigned off = cb + (unsigned)__float_as_int(tr) * P;
                        if (FALLBACK) return __ldg(reinterpret_cast<const float2*>(tvb + off));
#ifdef XR_DEBUG_BOUNDS
                        return *reinterpret_cast<const float2*>(sbase + XR_BOUND((long long)off, 0, (long long)box_bytes - 8));
#else
                        return *reinterpret_cast<const float2*>(sbase + off);
#endif
                    };
                    const float wk = __fdividef(wf * lf, fib);
                    const bool inside = (ub >= in_lo) && (ut <= in_hi);
                    float gprev = 0.0f;
                    if (__all_sync(__activemask(), inside)) {
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
                        const float ulo = lo_d - r0f, uhi = hi_d - r0f;
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
        } while (false);
        if (!FALLBACK) {
            // all threads are done with stage v % PS_NS: it takes view v + PS_NS
            __syncthreads();
            const int vn = v + PS_NS;
            if (vn < nview && vn % PS_WCH == 0) {
                windows(vn);
                __syncthreads();
            }
            if (tid == 0 && vn < nview && !*abort) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(vn);
                last = vn;
            }
        } else if ((v + 1) % PS_WCH == 0 && v + 1 < nview) {
            __syncthreads();
            windows(v + 1);
            __syncthreads();
        }
    }
    if (!FALLBACK) {
        __syncthreads();
        // every wait ended before this barrier, so all threads read the same
        if (*abort) {
            // the copies of the last PS_NS views issued may still be in flight
            if (tid == 0)
                for (int vp = max(last - (PS_NS - 1), 0); vp <= last; ++vp) {
                    const int4 wv = window_of(vp);
                    if (wv.x >= 0 && wv.z <= wv.w) mbar_wait_bounded(&bar[vp % PS_NS], (unsigned)((vp / PS_NS) & 1));
                }
            return;
        }
        if (tid == 0) unfit[cta] = s_unfit;
    }
    if (!active) return;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = j0 + i;
        if (j < g.D) st(vol + (((size_t)b * g.D + j) * g.H + iy) * g.W + ix, acc[i]);
    }
}

}  // namespace xr
