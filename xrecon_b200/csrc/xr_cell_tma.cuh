// Cell gather (A, B^T, Bw^T) with TMA-staged line windows.
//
// CTA = (view, 32 consecutive detector columns in traversal order, a group of
// NW*R detector rows).  Lane = column, warp = run of R rows.  The CTA sweeps
// the image lines; for every line the voxels its rays can touch form a window
// [p0, p0+BP) x [z0, z0+BZ) of (pixel along the line) x (z) that a single
// thread loads with one tiled TMA box (double buffered, one line ahead of
// the consumers; out-of-volume coordinates arrive as zeros).  Each thread then
// merges the z voxels of its column's pixel band against its R rows from
// shared memory, without bounds checks.  A line whose window does not fit the
// box (only for geometries far from the planned ones) falls back to global
// loads for that line.
//
// The window is a uniform function of the line index, evaluated identically
// by the producer thread (for line L+2) and by every consumer (for line L):
//   pixels: floor(pos_k0(L)) rounded down to a multiple of 8 (the TMA
//           alignment of the innermost coordinate) .. ceil(pos_kend(L)) - 1,
//   z:      floor(min t) .. floor(max t) over the CTA's columns and rows,
//           t = Q_k q(L) zd_r - z0/dz, extremes at Qmin/Qmax and the group's
//           first/last row boundary.
#pragma once

#include "xr_kernels.cuh"
#include "xr_tma.cuh"

namespace xr {

template <typename TI>
__device__ __forceinline__ float lds(const TI* p);
template <> __device__ __forceinline__ float lds<float>(const float* p) { return *p; }
template <> __device__ __forceinline__ float lds<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }
template <> __device__ __forceinline__ float lds<__half>(const __half* p) { return __half2float(*p); }

template <typename TI, int NB>
__device__ __forceinline__ float band_smem(const TI* p, const float (&w)[NB], int np) {
    float s = w[0] * lds(p);
#pragma unroll
    for (int i = 1; i < NB; ++i)
        if (i < np) s = fmaf(w[i], lds(p + i), s);
    return s;
}

// Elements of one stage of the TMA cell gather: BZ + 1 rows of BP, rounded
// up to 128 bytes.
template <typename TI>
__host__ __device__ inline int cell_stage_elems(int BP, int BZ) {
    return (int)(((size_t)BP * (BZ + 1) * sizeof(TI) + 127) / 128 * 128 / sizeof(TI));
}

struct CellWindow {
    int p0, z0, zlast, empty, ok;
};

struct CellCtaGeo {
    double bAk0, bBk0, bAke, bBke;  // first / last boundary of the CTA's columns
    double Qmin, Qmax;              // extremes of Q_k over the CTA's columns
    double zlo, zhi;                // unmagnified z of the row group's first / last boundary
};

// Window of line L, clamped to the image: pixels [0, npix), z [-1, D] (the
// rows -1 and D arrive as zeros from the TMA out-of-bounds fill and bound the
// voxel walks).  One voxel of margin on each side of the z range absorbs
// rounding between the window bound and each thread's own t values.
__host__ __device__ inline CellWindow cell_window(const CellCtaGeo& c, const ViewHdr& h, int L, double z0dz,
                                                  int npix, int D, int BP, int BZ) {
    CellWindow w;
    w.ok = 1;
    w.empty = 0;
    const double pl = fma(c.bBk0, (double)L, c.bAk0);
    const double ph = fma(c.bBke, (double)L, c.bAke);
    const double q = fma(h.q1, (double)L, h.q0);
    const double g0 = c.Qmin * q, g1 = c.Qmax * q;
    const double a0 = g0 * c.zlo, a1 = g1 * c.zlo, b0 = g0 * c.zhi, b1 = g1 * c.zhi;
    const double tl = fmin(fmin(a0, a1), fmin(b0, b1)) - z0dz;
    const double th = fmax(fmax(a0, a1), fmax(b0, b1)) - z0dz;
    if (!(pl > -1.0e8 && ph < 1.0e8 && tl > -1.0e8 && th < 1.0e8)) {
        w.p0 = w.z0 = w.zlast = 0;
        w.ok = 0;
        return w;
    }
    const int plo = max((int)floor(pl), 0);
    const int phi = min((int)ceil(ph) - 1, npix - 1);
    w.p0 = plo & ~7;
    w.z0 = max((int)floor(tl) - 1, -1);
    w.zlast = min((int)floor(th) + 1, D);
    w.empty = (plo > phi) || (w.z0 > w.zlast);
    w.ok = !w.empty && (phi - w.p0 < BP) && (w.zlast - w.z0 + 1 <= BZ);
    return w;
}

// Stages of the line ring; the block barrier that frees a stage comes after
// every XR_CELL_STAGES / 2 lines.
#ifndef XR_CELL_STAGES
#define XR_CELL_STAGES 4
#endif
constexpr int CELL_NS = XR_CELL_STAGES;
static_assert(CELL_NS == 2 || CELL_NS == 4, "two or four stages");
#ifndef XR_CELL_BATCH
#define XR_CELL_BATCH (XR_CELL_STAGES / 2)  // lines per block barrier
#endif
static_assert(XR_CELL_BATCH >= 1 && XR_CELL_BATCH < XR_CELL_STAGES, "a barrier frees at most all but one stage");

// After a wait gave up: only the last CELL_NS lines issued, up to `last`,
// may still have copies in flight (each earlier line's copy was seen to land
// by the issuing thread before it issued the next line into that stage).
// The issuing thread lets them land, or gives up once more, before the CTA
// exits, which keeps its shared memory allocated until then.
__device__ __noinline__ void drain_stages(uint64_t* bar, int last) {
    for (int Lp = max(last - (CELL_NS - 1), 0); Lp <= last; ++Lp)
        mbar_wait_bounded(&bar[Lp % CELL_NS], (unsigned)((Lp / CELL_NS) & 1));
}

// FINE: the geometry's detector rows are (nearly) all shorter than a voxel,
// so only the fine-row walk is compiled; lines where it does not apply take
// the global path.  Less code and fewer live registers than the full kernel.
#ifndef XR_CELL_MINB
#define XR_CELL_MINB 2  // CTAs per SM the register budget is sized for
#endif
#ifndef XR_CELL_VGROUP
#define XR_CELL_VGROUP 8  // views per group of the block order (below)
#endif
//
// HEL: helical scan, the view's z placement and column width come from
// vt.hel (the volume and detector rows measured from the view's source z).
// With MODE OP_BWT the helical weighted backprojection's transpose takes the
// column width cw_p (SOD du) and weighs slice j of view v by
// zwt[(j + 1) * nview + v] (rows -1 .. D + 1 of the table; the outer ones
// are zero).
template <typename TI, typename TO, int R, int NB, int MODE, bool FINE, bool HEL = false>
__global__ void __launch_bounds__(256, XR_CELL_MINB)
cell_tma3d_kernel(const Geom g, const ViewTables vt, const __grid_constant__ CUtensorMap map_rows,
                  const __grid_constant__ CUtensorMap map_cols, const TI* __restrict__ fb_rows,
                  const TI* __restrict__ fb_cols, const int pitch_rows, const int pitch_cols,
                  TO* __restrict__ sino, const int nview, const int view0, const double z0dz_p,
                  const double zd0_p, const double dvv, const float cw_p, const int BP, const int BZ,
                  const float* __restrict__ zwt) {
    constexpr bool ZW = HEL && MODE == OP_BWT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // each stage starts on a 128-byte boundary (TMA destination alignment) and
    // holds BZ + 1 rows: the spare row absorbs the look-ahead read of the
    // branch-free walk (never used in a result)
    const int stage_elems = cell_stage_elems<TI>(BP, BZ);
    TI* stage = reinterpret_cast<TI*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + (size_t)CELL_NS * stage_elems * sizeof(TI));
    // window of every line of this CTA (computed once, below)
    int4* wins = reinterpret_cast<int4*>(bar + CELL_NS);

    const int lane = threadIdx.x, tid = threadIdx.y * 32 + threadIdx.x;
    const int Nu = g.Nu;
    // Block order: XR_CELL_VGROUP consecutive views of each (column block,
    // row block) run next to each other, so that their nearly equal line
    // windows are read from DRAM once and from L2 after.
    unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    if (XR_CELL_VGROUP > 1) {
        const unsigned nx = gridDim.x, ny = gridDim.y, nz = gridDim.z;
        const unsigned id = blockIdx.x + nx * (blockIdx.y + ny * blockIdx.z);
        const unsigned grp = id / (XR_CELL_VGROUP * nx * ny), rem = id % (XR_CELL_VGROUP * nx * ny);
        const unsigned gsize = min((unsigned)XR_CELL_VGROUP, nz - grp * XR_CELL_VGROUP);  // the last group may be short
        bz = grp * XR_CELL_VGROUP + rem % gsize;
        bx = (rem / gsize) % nx;
        by = (rem / gsize) / nx;
    }
    const int k0 = (int)bx * 32;
    const int k = k0 + lane;
    const int kc = min(k, Nu - 1);
    const int rows_per_cta = blockDim.y * R;
    const int rg0 = (int)by * rows_per_cta;
    const int r0 = rg0 + threadIdx.y * R;
    const int vb = (int)bz + view0;
    const int v = vb % nview, b = vb / nview;
    const bool active = (k < Nu) && (r0 < g.Nv);

    const ViewHdr h = vt.hdr[v];
    const double z0dz = HEL ? vt.hel[v].z0dz : z0dz_p;
    const double zd0 = HEL ? vt.hel[v].zd0 : zd0_p;
    const float cw = (HEL && !ZW) ? vt.hel[v].cw : cw_p;
    // per-slice weight of this view (helical Bw^T): slice j at wz[(j + 1) * nview]
    const float* __restrict__ wz = ZW ? zwt + v : nullptr;
    auto slice_w = [&](int j) -> float { return ZW ? __ldg(wz + (size_t)(j + 1) * nview) : 1.0f; };
    const int use_x = h.use_x, nlines = h.nlines, npix = h.npix;
    const size_t ob = (size_t)v * (Nu + 1);
    const double bA0 = vt.bA[ob + kc], bB0 = vt.bB[ob + kc];
    const double bA1 = vt.bA[ob + kc + 1], bB1 = vt.bB[ob + kc + 1];
    const double Qk = vt.colQ[(size_t)v * Nu + kc];

    CellCtaGeo cg;
    {
        const int kend = min(k0 + 32, Nu);
        cg.bAk0 = vt.bA[ob + k0];
        cg.bBk0 = vt.bB[ob + k0];
        cg.bAke = vt.bA[ob + kend];
        cg.bBke = vt.bB[ob + kend];
        double qmn = Qk, qmx = Qk;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            qmn = fmin(qmn, __shfl_xor_sync(0xffffffffu, qmn, o));
            qmx = fmax(qmx, __shfl_xor_sync(0xffffffffu, qmx, o));
        }
        cg.Qmin = qmn;
        cg.Qmax = qmx;
        cg.zlo = zd0 + rg0 * dvv;
        cg.zhi = zd0 + (rg0 + rows_per_cta) * dvv;
    }
    const CUtensorMap* map = use_x ? &map_rows : &map_cols;
    const TI* __restrict__ fb = use_x ? fb_rows : fb_cols;
    const int pitch = use_x ? pitch_rows : pitch_cols;
    const size_t fb_plane = (size_t)nlines * pitch;
    const TI* __restrict__ fbb = fb + (size_t)b * g.D * fb_plane;
    const unsigned box_bytes = (unsigned)((size_t)BP * BZ * sizeof(TI));

    // test hook: arm the barrier for a box but issue no copy (the consumers'
    // bounded waits then run out with nothing in flight)
    const bool stall = (*(volatile unsigned*)&g_test_hooks & XR_HOOK_TMA_STALL) != 0;
    auto issue = [&](int L, int s) {
        const int4 w = wins[L];
        if (w.w >> 1) {
            mbar_arrive_expect_tx(&bar[s], box_bytes);
            if (!stall) tma_load_4d(stage + (size_t)s * stage_elems, map, w.x, L, w.y, b, &bar[s]);
        } else {
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&bar[s])) : "memory");
        }
    };
    // Set (0 -> 1, never back) by a wait that runs out.  Waits that find it
    // set give up at once, no further line is issued, nothing is stored.
    __shared__ int s_abort;
    volatile int* abort = &s_abort;
    if (tid == 0) {
        for (int i = 0; i < CELL_NS; ++i) mbar_init(&bar[i], 1);
        fence_barrier_init();
        s_abort = 0;
    }
    // the line windows, evaluated by all threads in parallel (FP64)
    for (int L = tid; L < nlines; L += blockDim.x * blockDim.y) {
        const CellWindow w = cell_window(cg, h, L, z0dz, npix, g.D, BP, BZ);
        wins[L] = make_int4(w.p0, w.z0, w.zlast, w.empty | (w.ok << 1));
    }
    // The spare row BZ of each stage is never written by TMA; the look-ahead
    // read multiplies it by zero, so it must hold finite values (zeros).
    for (int i = tid; i < CELL_NS * BP; i += blockDim.x * blockDim.y)
        stage[(size_t)(i / BP) * stage_elems + (size_t)BZ * BP + (i % BP)] = TI(0.0f);
    __syncthreads();
    int last = -1;  // last line issued (issuing thread)
    if (tid == 0)
        for (int L = 0; L < min(CELL_NS, nlines); ++L) issue(L, L), last = L;

    float acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = 0.0f;
    const double zr0 = zd0 + r0 * dvv;
    const float dpdz = (float)(h.dpix * g.dz);
    // Per-line terms, affine in the line L (q = q0 + q1 L): the run's first
    // row in slice units t0 = Qk q zr0 - z0dz (FP64: its floor and fraction
    // place every row), rows per slice bt = Qk q dvv and q itself for the
    // line factor (FP32, rounded as the kernel uses them).
    const double t0c = fma(Qk * h.q0, zr0, -z0dz), t0l = Qk * h.q1 * zr0;
    // Bw^T: the FBP weight of pixel p on line L.  The pixel centre is affine
    // in (L, p), so the flat detector's distance term R - (s . x) / R and the
    // arc detector's source offset are FMAs of L and p from per-view
    // constants (FP64, rounded once).
    float bw0 = 0.0f, bwL = 0.0f, bwp = 0.0f, bv0 = 0.0f, bvL = 0.0f, bvp = 0.0f;
    if (MODE == OP_BWT) {
        const double ax = (0.5 - 0.5 * g.W) * g.dx + g.shx;
        const double ay = (h.use_x ? (0.5 * g.H - 0.5) : (0.5 - 0.5 * g.H)) * g.dy + g.shy;
        const double bxL = h.use_x ? 0.0 : g.dx, bxp = h.use_x ? g.dx : 0.0;
        const double byL = h.use_x ? -g.dy : 0.0, byp = h.use_x ? 0.0 : g.dy;
        if (g.type == GEO_FLAT) {
            const double R = g.sod;
            bw0 = (float)(R - (h.sx * ax + h.sy * ay) / R);
            bwL = (float)(-(h.sx * bxL + h.sy * byL) / R);
            bwp = (float)(-(h.sx * bxp + h.sy * byp) / R);
        } else if (g.type == GEO_ARC) {
            bw0 = (float)(h.sx - ax); bwL = (float)(-bxL); bwp = (float)(-bxp);
            bv0 = (float)(h.sy - ay); bvL = (float)(-byL); bvp = (float)(-byp);
        }
    }
    auto bwt_weight = [&](float Lf, int pix) -> float {
        const float pf = (float)pix;
        if (g.type == GEO_FLAT) {
            const float R = (float)g.sod;
            const float den = fmaf(bwp, pf, fmaf(bwL, Lf, bw0));
            return __fdividef(R * R, den * den);
        }
        if (g.type == GEO_ARC) {
            const float ex = fmaf(bwp, pf, fmaf(bwL, Lf, bw0)), ey = fmaf(bvp, pf, fmaf(bvL, Lf, bv0));
            return __fdividef(1.0f, fmaf(ex, ex, ey * ey));
        }
        return 1.0f;
    };
    const float btc = (float)(Qk * dvv * h.q0), btl = (float)(Qk * dvv * h.q1);
    const float qc = (float)h.q0, ql = (float)h.q1;

    // After a wait gave up, the CTA still walks its remaining lines (every
    // read stays inside the staged windows, whatever they hold) so that all
    // threads meet every barrier; the results are dropped at the end.
    for (int L = 0; L < nlines; ++L) {
        const int s = L % CELL_NS;
        const unsigned parity = (unsigned)((L / CELL_NS) & 1);
        mbar_wait_bounded(&bar[s], parity, abort);
        CellWindow win;
        {
            const int4 wi = wins[L];
            win.p0 = wi.x; win.z0 = wi.y; win.zlast = wi.z; win.empty = wi.w & 1; win.ok = wi.w >> 1;
        }
        if (active) {
            const double pk = fma(bB0, (double)L, bA0);
            const double pk1 = fma(bB1, (double)L, bA1);
            const int pa = max((int)floor(pk), 0);
            const int pb = min((int)ceil(pk1) - 1, npix - 1);
            const float Lf = (float)L;
            const double t0 = fma(t0l, (double)L, t0c);
            const float bf = fmaf(btl, Lf, btc);
            const bool live = !win.empty && (pa <= pb) && (bf > 1.0e-4f && bf < 1.0e4f) &&
                              !(t0 + R * (double)bf <= 0.0 || t0 >= (double)g.D);
            if (live) {
                const double jf = floor(t0);
                const int j0 = (int)jf;
                const float f = (float)(t0 - jf);
                float lf = cw;
                if (MODE == OP_A) {
                    const float qf = fmaf(ql, Lf, qc);
                    lf = __fdividef(dpdz, qf * qf);
                }
                const float u0 = (float)(pk - (double)pa), u1 = (float)(pk1 - (double)pa);
                for (int pc = pa; pc <= pb; pc += NB) {
                    const int np = min(NB, pb - pc + 1);
                    const float off = (float)(pc - pa);
                    float w[NB];
#pragma unroll
                    for (int i = 0; i < NB; ++i) {
                        float wi = 0.0f;
                        if (i < np) {
                            wi = (fminf(off + (float)(i + 1), u1) - fmaxf(off + (float)i, u0)) * lf;
                            if (MODE == OP_BWT) wi *= bwt_weight(Lf, pc + i);
                        }
                        w[i] = wi;
                    }
                    float pos = f, jn = 1.0f, vj;
                    if (win.ok && bf < 0.999f) {
                        // Rows shorter than a voxel: each row crosses at most
                        // one voxel boundary.  In window slice coordinates
                        // u = t - (win.z0 - j0) (staged row = floor u), row i
                        // spans [u_i, u_{i+1}]; with n = floor(u_{i+1}) its
                        // part below n lies in slice n - 1, the slice of the
                        // previous row's top, and the rest in slice n:
                        //   row_i = band(n - 1) max(0, n - u_i)
                        //         + band(n) (u_{i+1} - max(n, u_i)).
                        // When the row does not cross, the first term is zero
                        // whatever band(n - 1) is, so each row forms one band
                        // and keeps it for the next; floor is a conversion
                        // to int and back (two issue slots; the rounding by
                        // an FP32 add of 1.5 * 2^23 took four and made the
                        // walk 5 % slower).  u is clamped to the staged
                        // slices 0 .. win.zlast - win.z0 (slices -1 and D of
                        // the volume arrive as zeros, and the window covers
                        // every t of the CTA otherwise).
                        const float fu = f + (float)(j0 - win.z0);
                        const float uhi = (float)(win.zlast - win.z0) + 0.999f;
                        const TI* sb = stage + (size_t)s * stage_elems + XR_BOUND(pc - win.p0, 0, BP - np);
                        auto slice_at = [&](float u, float& n) -> float {
                            const int ri = __float2int_rd(u);
                            n = (float)ri;
                            return band_smem<TI, NB>(sb + XR_BOUND(ri, 0, BZ) * BP, w, np) * slice_w(win.z0 + ri);
                        };
                        float up = fminf(fmaxf(fu, 0.0f), uhi);
                        float np0;
                        float bp = slice_at(up, np0);
#pragma unroll
                        for (int i = 0; i < R; ++i) {
                            const float u1 = fminf(fmaxf(fmaf(bf, (float)(i + 1), fu), 0.0f), uhi);
                            float n;
                            const float bn = slice_at(u1, n);
                            // max(0, n - u_i) = max(n, u_i) - u_i exactly
                            const float m = fmaxf(n, up);
                            acc[i] = fmaf(bp, m - up, acc[i]);
                            acc[i] = fmaf(bn, u1 - m, acc[i]);
                            bp = bn;
                            up = u1;
                        }
                    } else if (!FINE && win.ok) {
                        // Staged voxels win.z0 .. win.zlast; below the window a
                        // single virtual zero voxel ends at win.z0, past
                        // win.zlast the value is zero and the next boundary
                        // infinite.
                        const TI* sbase = stage + (size_t)s * stage_elems + XR_BOUND(pc - win.p0, 0, BP - np);
                        const TI* ptr;
                        int jabs;
                        if (j0 >= win.z0) {
                            jabs = j0;
                            ptr = sbase + (size_t)XR_BOUND(j0 - win.z0, 0, BZ) * BP;
                            vj = band_smem<TI, NB>(ptr, w, np) * slice_w(jabs);
                        } else {
                            jabs = win.z0 - 1;
                            ptr = sbase - BP;  // address only, advanced before any read
                            vj = 0.0f;
                            jn = (float)(win.z0 - j0);
                        }
#pragma unroll
                        for (int i = 0; i < R; ++i) {
                            const float top = fmaf(bf, (float)(i + 1), f);
                            float a = 0.0f;
                            while (jn < top) {
                                a = fmaf(jn - pos, vj, a);
                                pos = jn;
                                ++jabs;
                                ptr += BP;
#ifdef XR_DEBUG_BOUNDS
                                if (jabs <= win.zlast) ptr = sbase + (size_t)XR_BOUND(jabs - win.z0, 0, BZ) * BP;
#endif
                                if (jabs <= win.zlast) { vj = band_smem<TI, NB>(ptr, w, np) * slice_w(jabs); jn += 1.0f; }
                                else { vj = 0.0f; jn = 3.0e38f; }
                            }
                            if (top > pos) { a = fmaf(top - pos, vj, a); pos = top; }
                            acc[i] += a;
                        }
                    } else {
                        // global fallback with bounds checks
                        const TI* base = fbb + (size_t)L * pitch + pc;
                        int j = j0;
                        vj = ((unsigned)j < (unsigned)g.D) ? band_at(base + (size_t)j * fb_plane, w, np) * slice_w(j) : 0.0f;
#pragma unroll
                        for (int i = 0; i < R; ++i) {
                            const float top = fmaf(bf, (float)(i + 1), f);
                            float a = 0.0f;
                            while (jn < top) {
                                a = fmaf(jn - pos, vj, a);
                                pos = jn;
                                ++j;
                                jn += 1.0f;
                                vj = ((unsigned)j < (unsigned)g.D) ? band_at(base + (size_t)j * fb_plane, w, np) * slice_w(j) : 0.0f;
                            }
                            if (top > pos) { a = fmaf(top - pos, vj, a); pos = top; }
                            acc[i] += a;
                        }
                    }
                }
            }
        }
        // every BATCH lines: all warps are done with those lines' stages,
        // which take the lines CELL_NS further on
        constexpr int BATCH = XR_CELL_BATCH;
        if ((L + 1) % BATCH == 0) {
            __syncthreads();
            if (tid == 0 && !*abort) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                for (int j = L + 1 - BATCH; j <= L; ++j)
                    if (j + CELL_NS < nlines) issue(j + CELL_NS, j % CELL_NS), last = j + CELL_NS;
            }
        }
    }
    __syncthreads();
    // every wait ended before this barrier, so all threads read the same
    if (*abort) {
        if (tid == 0) drain_stages(bar, last);
        return;
    }

    if (!active) return;
    const int col = h.keep ? k : Nu - 1 - k;
    TO* out = sino + (((size_t)b * nview + v) * g.Nv) * Nu + col;
    float E = 1.0f, F = 0.0f, M = 0.0f;
    if (MODE == OP_A) {
        const size_t oc = (size_t)v * Nu + k;
        E = vt.colE[oc]; F = vt.colF[oc]; M = vt.colM[oc];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int r = r0 + i;
        if (r < g.Nv) {
            float sv = acc[i];
            if (MODE == OP_A) {
                float zc = (float)(zd0 + (r + 0.5) * dvv) * M;
                if (HEL) zc += vt.hel[v].zsrc;  // helical: the row's absolute z
                sv *= E * sqrtf(F + zc * zc);
            }
            st(out + (size_t)r * Nu, sv);
        }
    }
}

}  // namespace xr
