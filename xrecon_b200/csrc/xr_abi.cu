// C ABI of libxrecon_b200.so: validation, workspace layout and launches.
// The declarations and the reference interface each call replaces are in
// include/xrecon_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>

#include <array>
#include <atomic>
#include <cstring>
#include <type_traits>
#include <map>
#include <mutex>
#include <vector>

#include "xr_cell_tma.cuh"
#include "xr_vox_prefix.cuh"
#include "xr_vox_stage.cuh"
#include "xr_ragged.cuh"
#include "xr_sysmat.cuh"
#include "xr_rebin.cuh"
#include "xr_helical.cuh"
#include "xr_fft_filter.cuh"
#include "xr_ctpd.hpp"
#include "../../include/xrecon_b200.h"


namespace xr {
namespace {

thread_local std::string g_last_error;

// Test hook: route every operator through the plain (non-TMA) kernels.
bool g_force_plain = false;
// Host copy of the test hooks (xr_test_hooks); the launch code reads bit 3.
unsigned g_host_hooks = 0;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// Kernels launched by this library (process-wide; every launch site is
// followed by exactly one check_cuda).
std::atomic<unsigned long long> g_launches{0};

int check_cuda(const char* what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(XR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return XR_OK;
}

bool finite_pos(double v) { return std::isfinite(v) && v > 0.0; }

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

size_t dtype_size(int dt) { return dt == DT_F32 ? 4 : 2; }

bool dtype_ok(int dt) { return dt == DT_F32 || dt == DT_BF16 || dt == DT_F16; }

// Reject what the reference would silently turn into NaN/inf; everything
// the reference accepts with a finite result is accepted.
int validate(const Geom& g, int dim3d, int op, int nbatch, int nview) {
    if (op < 0 || op > 5) return fail(XR_ERR_INVALID_ARGUMENT, "unknown operator %d", op);
    if (g.type < GEO_PARALLEL || g.type > GEO_ARC)
        return fail(XR_ERR_INVALID_ARGUMENT, "scan type must be 0 (parallel), 1 (flat) or 2 (arc), got %d", g.type);
    if (g.W < 1 || g.H < 1 || g.D < 1 || g.Nu < 1 || g.Nv < 1)
        return fail(XR_ERR_INVALID_ARGUMENT, "image and detector sizes must be >= 1 (W=%d H=%d D=%d Nu=%d Nv=%d)",
                    g.W, g.H, g.D, g.Nu, g.Nv);
    if (!finite_pos(g.dx) || !finite_pos(g.dy) || !finite_pos(g.dz) || !finite_pos(g.du) || !finite_pos(g.dv))
        return fail(XR_ERR_INVALID_ARGUMENT, "pixel and detector spacings must be finite and > 0");
    if (!std::isfinite(g.shx) || !std::isfinite(g.shy) || !std::isfinite(g.shz) ||
        !std::isfinite(g.shu) || !std::isfinite(g.shv))
        return fail(XR_ERR_INVALID_ARGUMENT, "shifts must be finite");
    if (g.type != GEO_PARALLEL) {
        if (!finite_pos(g.sod) || !finite_pos(g.sdd))
            return fail(XR_ERR_INVALID_ARGUMENT, "fan/cone geometry needs finite iso_source > 0 and source_detector > 0");
        // The source must lie outside the image: the line magnification
        // S/(S - p) is only finite there.
        const double hx = 0.5 * g.W * g.dx + std::fabs(g.shx);
        const double hy = 0.5 * g.H * g.dy + std::fabs(g.shy);
        if (g.sod <= std::sqrt(hx * hx + hy * hy))
            return fail(XR_ERR_INVALID_ARGUMENT, "iso_source (%g) must exceed the image half-diagonal (%g)",
                        g.sod, std::sqrt(hx * hx + hy * hy));
        if (g.type == GEO_ARC && !(g.du * g.Nu < 3.0))
            return fail(XR_ERR_INVALID_ARGUMENT, "arc detector fan (Nu*du = %g rad) must be below pi", g.du * g.Nu);
    }
    if (dim3d) {
        // detector row height over voxel height on the common axis; the
        // kernels' merge loops assume it is a sane O(1) ratio.
        const double rs = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
        const double ratio = g.dv * rs / g.dz;
        if (!(ratio > 1e-3 && ratio < 1e3))
            return fail(XR_ERR_INVALID_ARGUMENT, "detector row / voxel height ratio %g outside [1e-3, 1e3]", ratio);
        if ((long long)g.D * nbatch > 65535)
            return fail(XR_ERR_UNSUPPORTED, "depth x batch (%lld) above 65535", (long long)g.D * nbatch);
    }
    if (nbatch < 1) return fail(XR_ERR_INVALID_ARGUMENT, "batch (B*C) must be >= 1");
    if (nview < 0) return fail(XR_ERR_INVALID_ARGUMENT, "number of views must be >= 0");
    (void)dim3d;
    return XR_OK;
}

Geom geom_from(const xr_geom3d* p) {
    Geom g;
    g.W = p->W; g.H = p->H; g.D = p->D; g.Nu = p->Nu; g.Nv = p->Nv; g.type = p->type;
    g.dx = p->dx; g.dy = p->dy; g.dz = p->dz; g.shx = p->shift_x; g.shy = p->shift_y; g.shz = p->shift_z;
    g.du = p->du; g.dv = p->dv; g.shu = p->shift_u; g.shv = p->shift_v; g.sod = p->sod; g.sdd = p->sdd;
    return g;
}

Geom geom_from(const xr_geom2d* p) {
    Geom g;
    g.W = p->W; g.H = p->H; g.D = 1; g.Nu = p->Nu; g.Nv = 1; g.type = p->type;
    g.dx = p->dx; g.dy = p->dy; g.dz = 1.0; g.shx = p->shift_x; g.shy = p->shift_y; g.shz = 0.0;
    g.du = p->du; g.dv = 1.0; g.shu = p->shift_u; g.shv = 0.0; g.sod = p->sod; g.sdd = p->sdd;
    return g;
}

struct Layout {
    size_t hdr, bA, bB, colQ, colR, colE, colF, colM, arc, colWR, volT, volR, volF, sinoS, pfxF, total;
    bool has_arc, has_pfx;
};

// Voxel-driven operators on a circular arc detector walk chained float32
// boundary angles, which need the per-boundary entries of ViewTables::arc.
bool arc_chain_op(const Geom& g, int op) {
    return g.type == GEO_ARC && (op == OP_B || op == OP_BW || op == OP_BT || op == OP_BWT);
}

// ------------------------------------------------------ TMA staging plans

struct CellPlan {
    bool ok;
    int BP, BZ, R;
    bool fine;  // rows longer than a voxel are rare: the fine-only kernel
};

constexpr int CELL_NW = 8;

int cell_rows_per_thread(const Geom& g) { return g.Nv >= 128 ? 16 : 8; }

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Sizes the line window of the TMA cell gather for this geometry by
// evaluating the kernel's own window function over the CTAs of views sampled
// densely in angle (the window depends on the angle only through smooth
// functions; the 45-degree axis switches are sampled on both sides).  Cached
// per geometry.
CellPlan plan_cell(const Geom& g) {
    static std::mutex mu;
    static std::map<std::string, CellPlan> cache;
    const std::string key(reinterpret_cast<const char*>(&g), sizeof(Geom));
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    CellPlan p{false, 0, 0, cell_rows_per_thread(g), false};
    double coarse = 0.0, pairs = 0.0;
    const int RG = CELL_NW * p.R;
    const double uscale = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
    const double rs = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
    const double zd0 = (-0.5 * g.Nv * g.dv + g.shv) * rs, dvv = g.dv * rs;
    const double z0dz = (-0.5 * g.D * g.dz + g.shz) / g.dz;
    std::vector<double> A(g.Nu + 1), B(g.Nu + 1), Q(g.Nu);
    std::vector<double> angles;
    const int NS = 256;
    for (int i = 0; i < NS; ++i) angles.push_back(2.0 * M_PI * i / NS + 0.37 / NS);
    for (int i = 0; i < 8; ++i) {
        angles.push_back(M_PI / 4 * i + 1e-5);
        angles.push_back(M_PI / 4 * i - 1e-5);
    }
    int maxspan = 0;
    double maxnz = 0.0;
    for (double ang : angles) {
        ViewHdr h;
        make_view_hdr(g, (float)ang, h);
        for (int k = 0; k <= g.Nu; ++k) {
            const double D = boundary_axis(g, h, (double)k, uscale);
            boundary_line_coeffs(g, h, D, A[k], B[k]);
        }
        for (int k = 0; k < g.Nu; ++k) Q[k] = column_mag(g, h, k, uscale) / g.dz;
        {
            // row length in voxels bt = Q_k q(L) dvv, q linear in L: the
            // fraction of this view's (column, line) pairs with bt >= 0.999
            const double n = (double)h.nlines;
            for (int k = 0; k < g.Nu; ++k) {
                const double a0 = std::fabs(Q[k] * dvv * h.q0);
                const double a1 = std::fabs(Q[k] * dvv * (h.q0 + h.q1 * (n - 1.0)));
                double f;
                if (a0 >= 0.999 && a1 >= 0.999) f = 1.0;
                else if (a0 < 0.999 && a1 < 0.999) f = 0.0;
                else f = (std::max(a0, a1) - 0.999) / std::fabs(a1 - a0);
                coarse += f;
                pairs += 1.0;
            }
        }
        for (int k0 = 0; k0 < g.Nu; k0 += 32) {
            const int kend = std::min(k0 + 32, g.Nu);
            CellCtaGeo c;
            c.bAk0 = A[k0]; c.bBk0 = B[k0]; c.bAke = A[kend]; c.bBke = B[kend];
            c.Qmin = 1e300; c.Qmax = -1e300;
            for (int k = k0; k < kend; ++k) { c.Qmin = std::min(c.Qmin, Q[k]); c.Qmax = std::max(c.Qmax, Q[k]); }
            for (int rg0 = 0; rg0 < g.Nv; rg0 += RG) {
                c.zlo = zd0 + rg0 * dvv;
                c.zhi = zd0 + (rg0 + RG) * dvv;
                for (int L : {0, h.nlines - 1}) {
                    const CellWindow w = cell_window(c, h, L, z0dz, h.npix, g.D, 1 << 30, 1 << 30);
                    if (w.empty) continue;
                    const double ph = std::fma(c.bBke, (double)L, c.bAke);
                    const int phi = std::min((int)std::ceil(ph) - 1, h.npix - 1);
                    maxspan = std::max(maxspan, phi - w.p0 + 1);
                    maxnz = std::max(maxnz, (double)(w.zlast - w.z0 + 1));
                }
            }
        }
    }
    p.fine = pairs > 0.0 && coarse < 0.05 * pairs;
    p.BP = round_up(std::max(maxspan, 8), 8);
    p.BZ = (int)maxnz;
    p.ok = p.BP <= 256 && p.BZ <= 256 && p.BZ >= 1 &&
           (size_t)CELL_NS * p.BP * (p.BZ + 1) * 4 + (size_t)std::max(g.W, g.H) * 16 + 8 * CELL_NS <= 200 * 1024;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = p;
    return p;
}

using EncodeTiledFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    });
    return fn;
}

// 4D map over [nbatch][D][nlines][pitch] (pitch >= npix) with box (BP, 1, BZ, 1).
bool encode_line_map(CUtensorMap* m, int dt, const void* base, int npix, int nlines, int D, int nbatch, int pitch,
                     int BP, int BZ) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const size_t es = dt == DT_F32 ? 4 : 2;
    const CUtensorMapDataType t = dt == DT_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                : dt == DT_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    cuuint64_t dims[4] = {(cuuint64_t)npix, (cuuint64_t)nlines, (cuuint64_t)D, (cuuint64_t)nbatch};
    cuuint64_t strides[3] = {(cuuint64_t)pitch * es, (cuuint64_t)pitch * nlines * es,
                             (cuuint64_t)pitch * nlines * D * es};
    cuuint32_t box[4] = {(cuuint32_t)BP, 1u, (cuuint32_t)BZ, 1u};
    cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
    const CUresult r = fn(m, t, 4, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Image-input ops of the cell gather need the flipped transpose of the image
// (lines of y-axis views); cone A^T needs an FP32 pre-scaled sinogram.
#ifndef XR_PFX_R
#define XR_PFX_R 16
#endif
#ifndef XR_PFX_NWY
#define XR_PFX_NWY 8
#endif
constexpr int PFX_R = XR_PFX_R;  // z voxels per thread of the prefix backprojection

Layout layout(int dim3d, int op, const Geom& g, int nbatch, int nview, int dtype_in, bool chain_ok = true) {
    Layout l{};
    size_t o = 0;
    const size_t V = (size_t)(nview > 0 ? nview : 1);
    l.hdr = o;   o = align256(o + V * sizeof(ViewHdr));
    l.bA = o;    o = align256(o + V * (g.Nu + 1) * sizeof(double));
    l.bB = o;    o = align256(o + V * (g.Nu + 1) * sizeof(double));
    l.colQ = o;  o = align256(o + V * g.Nu * sizeof(double));
    l.colR = o;  o = align256(o + V * g.Nu * sizeof(double));
    l.colE = o;  o = align256(o + V * g.Nu * sizeof(float));
    l.colF = o;  o = align256(o + V * g.Nu * sizeof(float));
    l.colM = o;  o = align256(o + V * g.Nu * sizeof(float));
    l.has_arc = chain_ok && arc_chain_op(g, op);
    l.arc = o;
    if (l.has_arc) o = align256(o + 2 * V * (g.Nu + 1) * sizeof(float4));
    int eff = op;
    if (g.type == GEO_PARALLEL && dim3d) {
        if (op == OP_B || op == OP_BW) eff = OP_AT;
        else if (op == OP_BT || op == OP_BWT) eff = OP_A;
    }
    // the prefix gathers' FP32 column steps
    l.has_pfx = dim3d && (eff == OP_AT || eff == OP_B || eff == OP_BW);
    l.colWR = o;
    if (l.has_pfx) o = align256(o + V * g.Nu * sizeof(float4));
    l.volT = o;
    l.volR = o;
    if (eff == OP_A || eff == OP_BT || eff == OP_BWT) {
        // flipped transpose with a 16-byte-multiple pitch, plus (when the
        // input rows are not) a padded copy of the input rows.  3D images
        // stored in half precision are widened to FP32 once (volF) and
        // staged from there, so their transpose and rows are FP32 too.
        const bool widen = dim3d && dtype_size(dtype_in) == 2;
        const size_t es = widen ? 4 : dtype_size(dtype_in);
        o = align256(o + (size_t)nbatch * g.D * g.W * round_up(g.H, 8) * es);
        l.volR = o;
        if (dim3d && ((size_t)g.W * es) % 16 != 0)
            o = align256(o + (size_t)nbatch * g.D * g.H * round_up(g.W, 8) * es);
        l.volF = o;
        if (widen) o = align256(o + (size_t)nbatch * g.D * g.H * g.W * sizeof(float));
    }
    // voxel-gather ops: the per-view row prefix tables (float2, Nv + 2 rows);
    // the plain kernels' pre-scaled cone A^T sinogram reuses the region
    l.sinoS = o;
    if (dim3d && (eff == OP_AT || eff == OP_B || eff == OP_BW))
        o = align256(o + (size_t)nbatch * V * (g.Nv + 2) * g.Nu * sizeof(float2));
    // the staged prefix gather's per-CTA flags (views left to its fallback)
    l.pfxF = o;
    if (l.has_pfx)
        o = align256(o + (size_t)((g.W + PS_T - 1) / PS_T) * ((g.H + PS_T - 1) / PS_T) *
                             ((g.D + PFX_R - 1) / PFX_R) * nbatch * sizeof(int));
    l.total = o;
    return l;
}

ViewTables tables_at(char* ws, const Layout& l) {
    ViewTables t;
    t.hdr = reinterpret_cast<ViewHdr*>(ws + l.hdr);
    t.bA = reinterpret_cast<double*>(ws + l.bA);
    t.bB = reinterpret_cast<double*>(ws + l.bB);
    t.colQ = reinterpret_cast<double*>(ws + l.colQ);
    t.colR = reinterpret_cast<double*>(ws + l.colR);
    t.colE = reinterpret_cast<float*>(ws + l.colE);
    t.colF = reinterpret_cast<float*>(ws + l.colF);
    t.colM = reinterpret_cast<float*>(ws + l.colM);
    t.hel = nullptr;
    t.arc = l.has_arc ? reinterpret_cast<float4*>(ws + l.arc) : nullptr;
    t.colWR = l.has_pfx ? reinterpret_cast<float4*>(ws + l.colWR) : nullptr;
    return t;
}

// Row boundaries of the detector before magnification: zd_r = zd0 + r*dvv
// (forward3d.cpp:318-320; flat rows live on the virtual detector).
void row_params(const Geom& g, double& zd0, double& dvv, double& z0dz) {
    const double rs = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
    zd0 = (-0.5 * g.Nv * g.dv + g.shv) * rs;
    dvv = g.dv * rs;
    z0dz = (-0.5 * g.D * g.dz + g.shz) / g.dz;
}

// Column width of the backprojection: flat du*SOD/SDD (3D) or du (2D,
// already scaled); arc 2*SOD*tan(du/2); parallel du (xrmath.h:188-198,
// backward2d.cpp:87,109,185).
float column_width(const Geom& g, int dim3d) {
    if (g.type == GEO_FLAT) return (float)(dim3d ? g.du * g.sod / g.sdd : g.du);
    if (g.type == GEO_ARC) return (float)(2.0 * g.sod * std::tan(0.5 * g.du));
    return (float)g.du;
}

GeomF make_geomf(const Geom& g, int dim3d) {
    GeomF f;
    f.x0 = (float)(-0.5 * g.W * g.dx + g.shx);
    f.y0 = (float)(-0.5 * g.H * g.dy + g.shy);
    f.xc0 = (float)((0.5 - 0.5 * g.W) * g.dx + g.shx);
    f.yc0 = (float)((0.5 * g.H - 0.5) * g.dy + g.shy);
    f.dx = (float)g.dx;
    f.dy = (float)g.dy;
    f.sod = (float)g.sod;
    f.uscale = (dim3d && g.type == GEO_FLAT) ? (float)(g.sod / g.sdd) : 1.0f;
    f.shu = (float)g.shu;
    f.du = (float)g.du;
    f.inv_uscale = 1.0f / f.uscale;
    f.inv_du = (float)(1.0 / g.du);
    f.H = g.H;
    f.Nu = g.Nu;
    f.type = g.type;
    return f;
}

// Box of the staged prefix gather (vox_stage3d_kernel), sized by evaluating
// its window over every tile and z-run of views sampled densely in angle
// (the windows are smooth functions of the angle; the 45-degree axis
// switches are sampled on both sides), with two columns and two rows to
// spare.  The box is capped at the shared memory that leaves room for four
// CTAs per SM (what 64 registers a thread allow): when the largest window
// does not fit that, the box takes the shape (columns x rows within the cap)
// that holds the most sampled windows, and the rest go to the fallback
// launch (about 3 % of (CTA, view) pairs on the 512-cube workload: B 155 ->
// 140 ms against the uncapped box at three CTAs per SM).  Cached per
// geometry.
struct PfxStagePlan {
    bool ok;
    int BC, BR;
};

PfxStagePlan plan_pfx_stage(const Geom& g) {
    static std::mutex mu;
    static std::map<std::string, PfxStagePlan> cache;
    const std::string key(reinterpret_cast<const char*>(&g), sizeof(Geom));
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    PfxStagePlan p{false, 0, 0};
    if ((g.type == GEO_FLAT || g.type == GEO_PARALLEL || g.type == GEO_ARC) && g.Nu % 2 == 0 &&
        (g.type != GEO_ARC || XR_GUESS_ATAN_ERR / g.du < 0.25)) {
        const GeomF gf = make_geomf(g, 1);
        double zd0, dvv, z0dz;
        {
            const double rs = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
            zd0 = (-0.5 * g.Nv * g.dv + g.shv) * rs;
            dvv = g.dv * rs;
            z0dz = (-0.5 * g.D * g.dz + g.shz) / g.dz;
        }
        const double zoffh = -zd0 / dvv - 0.5;
        const double uscale = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
        std::vector<double> angles;
        for (int i = 0; i < 256; ++i) angles.push_back(2.0 * M_PI * i / 256 + 0.37 / 256);
        for (int i = 0; i < 8; ++i) {
            angles.push_back(M_PI / 4 * i + 1e-5);
            angles.push_back(M_PI / 4 * i - 1e-5);
        }
        int maxc = 0, maxr = 0;
        bool bad = false;
        // windows sampled, by (columns, rows) needed; 257 = more than a box holds
        std::vector<double> hist(258 * 258, 0.0);
        double nsamp = 0.0;
        for (double ang : angles) {
            ViewHdr h;
            make_view_hdr(g, (float)ang, h);
            auto colk = [&](double x, double y) {  // fractional column (traversal order) of a point
                double sg;
                if (g.type == GEO_ARC) {
                    const double ex = x - h.sx, ey = y - h.sy;
                    sg = std::atan2(h.dcx * ey - h.dcy * ex, h.dcx * ex + h.dcy * ey) / g.du;
                } else if (g.type == GEO_FLAT) {
                    const double R = g.sod;
                    const double u = R * (x * h.c + y * h.s) / (R + x * h.s - y * h.c);
                    sg = (u / uscale - g.shu) / g.du;
                } else {
                    sg = (x * h.c + y * h.s - g.shu) / g.du;
                }
                return h.keep ? sg + 0.5 * g.Nu : 0.5 * g.Nu - sg;
            };
            auto colR = [&](int k) { return g.type == GEO_PARALLEL ? g.dz : g.dz / column_mag(g, h, k, uscale); };
            for (int iy0 = 0; iy0 < g.H; iy0 += PS_T)
                for (int ix0 = 0; ix0 < g.W; ix0 += PS_T) {
                    const int ixe = std::min(ix0 + PS_T, g.W) - 1, iye = std::min(iy0 + PS_T, g.H) - 1;
                    double xl, xr, yl, yh;
                    int L0, L1;
                    if (h.use_x) {
                        L0 = iy0; L1 = iye;
                        xl = gf.x0 + ix0 * (double)gf.dx; xr = gf.x0 + (ixe + 1) * (double)gf.dx;
                        yh = gf.yc0 - L0 * (double)gf.dy; yl = gf.yc0 - L1 * (double)gf.dy;
                    } else {
                        L0 = ix0; L1 = ixe;
                        xl = gf.xc0 + L0 * (double)gf.dx; xr = gf.xc0 + L1 * (double)gf.dx;
                        yl = gf.y0 + (g.H - 1 - iye) * (double)gf.dy; yh = gf.y0 + (g.H - iy0) * (double)gf.dy;
                    }
                    const double ks[4] = {colk(xl, yl), colk(xl, yh), colk(xr, yl), colk(xr, yh)};
                    double gmin = std::min(std::min(ks[0], ks[1]), std::min(ks[2], ks[3]));
                    double gmax = std::max(std::max(ks[0], ks[1]), std::max(ks[2], ks[3]));
                    gmin = std::max(std::min(gmin, g.Nu + 2.0), -2.0);
                    gmax = std::max(std::min(gmax, g.Nu + 2.0), -2.0);
                    // arc B / Bw (chained walk): widened by the brackets' half-width bound
                    double wm = 1.5;
                    if (g.type == GEO_ARC) {
                        const double ddx = std::max(std::max(xl - h.sx, h.sx - xr), 0.0);
                        const double ddy = std::max(std::max(yl - h.sy, h.sy - yh), 0.0);
                        const double a = 0.5 * (h.use_x ? gf.dx : gf.dy), rlo = std::sqrt(ddx * ddx + ddy * ddy);
                        wm += a / std::max(rlo - a, a) / g.du * 1.002;
                    }
                    const int kw0 = std::max(0, (int)std::floor(gmin - wm)), kw1 = std::min(g.Nu - 1, (int)std::floor(gmax + wm));
                    if (kw0 > kw1) continue;
                    const int c0 = (h.keep ? kw0 : g.Nu - 1 - kw1) & ~1, c1 = h.keep ? kw1 : g.Nu - 1 - kw0;
                    maxc = std::max(maxc, c1 - c0 + 1);
                    const int hc = std::min(257, c1 - c0 + 1 + 2);
                    const double d0 = std::fma(h.q1, (double)L0, h.q0) * dvv, d1 = std::fma(h.q1, (double)L1, h.q0) * dvv;
                    double slack = 0.0;
                    if (g.type == GEO_ARC) {
                        const double wd = (double)(kw1 - kw0 + 1) * g.du;
                        slack = 1.01 * g.dz * g.sdd / std::fabs(h.sperp) * wd * wd / 8.0 + 1e-12;
                    }
                    const double Rlo = std::min(colR(kw0), colR(kw1)) - slack, Rhi = std::max(colR(kw0), colR(kw1)) + slack;
                    if (!(d0 > 0.0 && d1 > 0.0 && Rlo > 0.0)) { bad = true; continue; }
                    const double ibmin = Rlo / std::max(d0, d1), ibmax = Rhi / std::min(d0, d1);
                    for (int j0 = 0; j0 < g.D; j0 += PFX_R) {
                        const double zs = j0 + z0dz, zt = zs + PFX_R;
                        const double ulo = zoffh + std::min(zs * ibmin, zs * ibmax);
                        const double uhi = zoffh + std::max(zt * ibmin, zt * ibmax);
                        if (!(ulo <= uhi) || ulo > g.Nv + 2.0 || uhi < -3.0) continue;
                        const int rlo = std::max(0, (int)std::floor(std::max(ulo, -4.0)));
                        const int rhi = std::min(g.Nv + 1, (int)std::ceil(std::min(uhi, g.Nv + 4.0)) + 2);
                        maxr = std::max(maxr, rhi - rlo + 1);
                        hist[hc * 258 + std::min(257, rhi - rlo + 1 + 2)] += 1.0;
                        nsamp += 1.0;
                    }
                }
        }
        int BC = round_up(std::max(maxc + 2, 8), 2);
        if (BC % 16 == 0) BC += 2;  // rows of the box then start on different banks
        int BR = maxr + 2;
        // 228 KB of shared memory per SM, 1 KB reserved per CTA
        auto ctas = [](int bc, int br) { return (int)((228 * 1024) / (pfx_stage_smem(bc, br) + 1024)); };
        bool fits_all = BC <= 256 && BR <= 256 && ctas(BC, BR) >= 4;
        if (!fits_all && nsamp > 0.0) {
            // fraction of sampled windows each box holds: 2D prefix counts
            std::vector<double> cum(258 * 258, 0.0);
            for (int c = 0; c < 258; ++c)
                for (int r = 0; r < 258; ++r)
                    cum[c * 258 + r] = hist[c * 258 + r] + (c ? cum[(c - 1) * 258 + r] : 0.0) +
                                       (r ? cum[c * 258 + r - 1] : 0.0) - (c && r ? cum[(c - 1) * 258 + r - 1] : 0.0);
            double best = -1.0;
            int bc_best = 0, br_best = 0;
            for (int bc = 8; bc <= 256; bc += 2) {
                if (bc % 16 == 0) continue;
                int br = 256;
                while (br > 0 && ctas(bc, br) < 4) --br;
                if (br < 1) continue;
                const double held = cum[bc * 258 + br];
                if (held > best) best = held, bc_best = bc, br_best = br;
            }
            // more than a tenth of the windows in the fallback: the uncapped
            // box at three CTAs per SM, if it fits that
            if (best >= 0.9 * nsamp) BC = bc_best, BR = br_best;
        }
        p.ok = !bad && maxc > 0 && maxr > 0 && BC <= 256 && BR <= 256 && ctas(BC, BR) >= 3;
        p.BC = BC;
        p.BR = BR;
    }
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = p;
    return p;
}

// 3D map over the row-prefix tables [batch x views][Nv + 2][Nu] of float2,
// read as 8-byte elements, with box (BC, BR, 1).
bool encode_table_map(CUtensorMap* m, const float2* tab, const Geom& g, int nbv, int BC, int BR) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)g.Nu, (cuuint64_t)(g.Nv + 2), (cuuint64_t)nbv};
    cuuint64_t strides[2] = {(cuuint64_t)g.Nu * 8, (cuuint64_t)g.Nu * 8 * (g.Nv + 2)};
    cuuint32_t box[3] = {(cuuint32_t)BC, (cuuint32_t)BR, 1u};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<float2*>(tab), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

constexpr int CELL_R = 8;
constexpr int VOX_R = 16;
constexpr int VOX_NW = 4;
constexpr int PFX_NWY = XR_PFX_NWY;  // image lines (warps) per CTA

template <typename T> constexpr int dtype_code();
template <> constexpr int dtype_code<float>() { return DT_F32; }
template <> constexpr int dtype_code<__nv_bfloat16>() { return DT_BF16; }
template <> constexpr int dtype_code<__half>() { return DT_F16; }

// Staged prefix gather (vox_stage3d_kernel), then its fallback launch for
// the views a CTA could not stage; -1 when this geometry is not covered (the
// caller then uses vox_prefix3d_kernel).
template <typename TO, int MODE, bool HEL, bool CHAIN = false>
int launch_pfx_stage_mode(const Geom& g, const GeomF& gf, const ViewTables& vt, const CUtensorMap& map,
                          const float2* tab, TO* out, int* flags, int nbatch, int nview, int nzp, int BC, int BR,
                          cudaStream_t st, double z0dz, double zd0, double dvv, float cw, float atconst, float oscale) {
    auto ks = vox_stage3d_kernel<TO, PFX_R, MODE, false, HEL, CHAIN>;
    auto kf = vox_stage3d_kernel<TO, PFX_R, MODE, true, HEL, CHAIN>;
    const size_t smem = pfx_stage_smem(BC, BR), smem_fb = 2 * PS_WCH * sizeof(int4) + 128;
    if (cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(XR_ERR_CUDA, "cannot reserve %zu bytes of shared memory", smem);
    const dim3 grid((g.W + PS_T - 1) / PS_T, (g.H + PS_T - 1) / PS_T, nzp * nbatch);
    ks<<<grid, PS_T * PS_T, smem, st>>>(g, gf, vt, map, tab, out, flags, nview, nzp, z0dz, zd0, dvv, cw, atconst,
                                        oscale, BC, BR);
    if (int rc = check_cuda("vox_stage3d")) return rc;
    kf<<<grid, PS_T * PS_T, smem_fb, st>>>(g, gf, vt, map, tab, out, flags, nview, nzp, z0dz, zd0, dvv, cw, atconst,
                                           oscale, BC, BR);
    return check_cuda("vox_stage3d (fallback)");
}

template <typename TO, bool HEL = false>
int run_pfx_stage(int eff, const Geom& g, const GeomF& gf, const ViewTables& vt, const float2* tab, TO* out,
                  int nbatch, int nview, int nzp, char* ws, const Layout& l, cudaStream_t st, double z0dz,
                  double zd0, double dvv, float cw, float atconst, float oscale) {
    const PfxStagePlan sp = plan_pfx_stage(g);
    if (!sp.ok) return -1;
    CUtensorMap map;
    if (!encode_table_map(&map, tab, g, nbatch * nview, sp.BC, sp.BR)) return -1;
    int* flags = reinterpret_cast<int*>(ws + l.pfxF);
    if (eff == OP_AT)
        return launch_pfx_stage_mode<TO, OP_AT, HEL>(g, gf, vt, map, tab, out, flags, nbatch, nview, nzp, sp.BC, sp.BR,
                                                     st, z0dz, zd0, dvv, cw, atconst, oscale);
    if (eff == OP_B && vt.arc && !HEL)
        return launch_pfx_stage_mode<TO, OP_B, false, true>(g, gf, vt, map, tab, out, flags, nbatch, nview, nzp, sp.BC,
                                                           sp.BR, st, z0dz, zd0, dvv, cw, atconst, oscale);
    if (eff == OP_B)
        return launch_pfx_stage_mode<TO, OP_B, HEL>(g, gf, vt, map, tab, out, flags, nbatch, nview, nzp, sp.BC, sp.BR,
                                                    st, z0dz, zd0, dvv, cw, atconst, oscale);
    if (HEL) return -1;  // the helical Bw is hel_wbp_kernel
    if (vt.arc)  // arc detector: the chained column walk
        return launch_pfx_stage_mode<TO, OP_BW, false, true>(g, gf, vt, map, tab, out, flags, nbatch, nview, nzp, sp.BC,
                                                            sp.BR, st, z0dz, zd0, dvv, cw, atconst, oscale);
    return launch_pfx_stage_mode<TO, OP_BW, HEL>(g, gf, vt, map, tab, out, flags, nbatch, nview, nzp, sp.BC, sp.BR, st,
                                                 z0dz, zd0, dvv, cw, atconst, oscale);
}

template <typename TI, typename TO, int R, int MODE, bool HEL>
int launch_cell_tma_mode(const Geom& g, const CellPlan& p, const CUtensorMap& mr, const CUtensorMap& mc,
                         const TI* rows, const TI* cols, int pitch_r, int pitch_c, TO* out, int nbatch, int nview,
                         const ViewTables& vt, cudaStream_t st, double z0dz, double zd0, double dvv, float cw,
                         const float* zwt) {
    auto kern = p.fine ? cell_tma3d_kernel<TI, TO, R, 2, MODE, true, HEL>
                       : cell_tma3d_kernel<TI, TO, R, 2, MODE, false, HEL>;
    const int maxlines = std::max(g.W, g.H);
    const size_t smem = CELL_NS * (size_t)cell_stage_elems<TI>(p.BP, p.BZ) * sizeof(TI) + 8 * CELL_NS +
                        (size_t)maxlines * sizeof(int4);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(XR_ERR_CUDA, "cannot reserve %zu bytes of shared memory", smem);
    const int RG = CELL_NW * R;
    const int total = nview * nbatch;
    for (int z0 = 0; z0 < total; z0 += 65535) {
        const int nz = std::min(65535, total - z0);
        dim3 grid((g.Nu + 31) / 32, (g.Nv + RG - 1) / RG, nz);
        kern<<<grid, dim3(32, CELL_NW), smem, st>>>(g, vt, mr, mc, rows, cols, pitch_r, pitch_c, out, nview, z0, z0dz,
                                                    zd0, dvv, cw, p.BP, p.BZ, zwt);
        if (int rc = check_cuda("cell_tma3d")) return rc;
    }
    return XR_OK;
}

// Cell gather with TMA line windows; returns -1 when this configuration is
// not covered (the caller then uses the plain kernel).
// Window plan of a helical scan: the views' z placement varies, so the z
// extent is sized on a volume deep enough that no window is clamped, then
// capped at the real depth (a window never spans more than D + 2 slices).
CellPlan plan_cell_helical(const Geom& g) {
    Geom gp = g;
    gp.D = 1 << 20;
    gp.shz = 0.0;
    CellPlan p = plan_cell(gp);
    p.BZ = std::min(p.BZ, g.D + 2);
    p.ok = p.ok && p.BZ >= 1;
    return p;
}

template <typename TI, typename TO, bool HEL = false>
int run_cell_tma(int eff, const Geom& g, const TI* in, TO* out, int nbatch, int nview, char* ws, const Layout& l,
                 const ViewTables& vt, cudaStream_t st, double z0dz, double zd0, double dvv, float cw,
                 const float* zwt = nullptr) {
    // FP32 images (also widened half-precision ones) go to any output type
    if (!std::is_same<TI, float>::value && !std::is_same<TO, TI>::value && !std::is_same<TO, float>::value)
        return -1;
    if (reinterpret_cast<uintptr_t>(in) % 16 != 0) return -1;
    const CellPlan p = HEL ? plan_cell_helical(g) : plan_cell(g);
    if (!p.ok || !encode_fn()) return -1;
    const size_t es = sizeof(TI);
    const int Hp = round_up(g.H, 8);
    TI* cols = reinterpret_cast<TI*>(ws + l.volT);
    dim3 tg((g.W + 31) / 32, (g.H + 31) / 32, g.D * nbatch);
    transpose_flip_kernel<TI><<<tg, dim3(32, 8), 0, st>>>(in, cols, g.H, g.W, Hp);
    if (int rc = check_cuda("transpose")) return rc;
    const TI* rows = in;
    int Wp = g.W;
    if (((size_t)g.W * es) % 16 != 0) {
        Wp = round_up(g.W, 8);
        TI* vr = reinterpret_cast<TI*>(ws + l.volR);
        const size_t nrows = (size_t)nbatch * g.D * g.H;
        const size_t n = nrows * g.W;
        pad_rows_kernel<TI><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, vr, g.W, Wp, nrows);
        if (int rc = check_cuda("pad_rows")) return rc;
        rows = vr;
    }
    CUtensorMap mr, mc;
    if (!encode_line_map(&mr, dtype_code<TI>(), rows, g.W, g.H, g.D, nbatch, Wp, p.BP, p.BZ) ||
        !encode_line_map(&mc, dtype_code<TI>(), cols, g.H, g.W, g.D, nbatch, Hp, p.BP, p.BZ))
        return -1;
    if (p.R == 16) {
        if (eff == OP_A) return launch_cell_tma_mode<TI, TO, 16, OP_A, HEL>(g, p, mr, mc, rows, cols, Wp, Hp, out, nbatch, nview, vt, st, z0dz, zd0, dvv, cw, zwt);
        if (eff == OP_BT) return launch_cell_tma_mode<TI, TO, 16, OP_BT, HEL>(g, p, mr, mc, rows, cols, Wp, Hp, out, nbatch, nview, vt, st, z0dz, zd0, dvv, cw, zwt);
        return launch_cell_tma_mode<TI, TO, 16, OP_BWT, HEL>(g, p, mr, mc, rows, cols, Wp, Hp, out, nbatch, nview, vt, st, z0dz, zd0, dvv, cw, zwt);
    }
    if (eff == OP_A) return launch_cell_tma_mode<TI, TO, 8, OP_A, HEL>(g, p, mr, mc, rows, cols, Wp, Hp, out, nbatch, nview, vt, st, z0dz, zd0, dvv, cw, zwt);
    if (eff == OP_BT) return launch_cell_tma_mode<TI, TO, 8, OP_BT, HEL>(g, p, mr, mc, rows, cols, Wp, Hp, out, nbatch, nview, vt, st, z0dz, zd0, dvv, cw, zwt);
    return launch_cell_tma_mode<TI, TO, 8, OP_BWT, HEL>(g, p, mr, mc, rows, cols, Wp, Hp, out, nbatch, nview, vt, st, z0dz, zd0, dvv, cw, zwt);
}

template <typename TI, typename TO>
int run3d(int op, const Geom& g, const TI* in, TO* out, const float* ang, int nbatch, int nview,
          char* ws, const Layout& l, cudaStream_t st, float oscale) {
    const ViewTables vt = tables_at(ws, l);
    double zd0, dvv, z0dz;
    row_params(g, zd0, dvv, z0dz);
    const float cw = column_width(g, 1);
    const size_t nvox = (size_t)g.D * g.H * g.W;
    if (nview == 0) {
        if (op == OP_AT || op == OP_B || op == OP_BW) {
            if (cudaMemsetAsync(out, 0, nvox * nbatch * sizeof(TO), st) != cudaSuccess)
                return fail(XR_ERR_CUDA, "memset failed");
        }
        return XR_OK;
    }
    {
        dim3 grid((g.Nu + 1 + 127) / 128, nview);
        setup_views_kernel<<<grid, 128, 0, st>>>(g, 1, ang, nview, vt);
        if (int rc = check_cuda("setup_views")) return rc;
    }
    int eff = op;
    if (g.type == GEO_PARALLEL) {
        if (op == OP_B || op == OP_BW) eff = OP_AT;
        else if (op == OP_BT || op == OP_BWT) eff = OP_A;
    }
    if (eff == OP_A || eff == OP_BT || eff == OP_BWT) {
        // arc B^T / Bw^T walk chained angles per pixel: the plain cell gather
        if (!g_force_plain && !vt.arc) {
            int rc;
            if constexpr (sizeof(TI) == 2) {
                // Widen once: the staged walk then reads FP32, which costs
                // fewer instructions than widening every staged read (the
                // values, and so the results, are the same)
                float* vf = reinterpret_cast<float*>(ws + l.volF);
                const size_t n = (size_t)nbatch * g.D * g.H * g.W;
                const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(vf)) & 15) == 0;
                const size_t nt = vec ? (n + 7) / 8 : n;
                widen_kernel<TI><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(in, vf, n, vec);
                if (int e = check_cuda("widen")) return e;
                rc = run_cell_tma<float, TO>(eff, g, vf, out, nbatch, nview, ws, l, vt, st, z0dz, zd0, dvv, cw);
            } else {
                rc = run_cell_tma(eff, g, in, out, nbatch, nview, ws, l, vt, st, z0dz, zd0, dvv, cw);
            }
            if (rc >= 0) return rc;
        }
        TI* volT = reinterpret_cast<TI*>(ws + l.volT);
        dim3 tg((g.W + 31) / 32, (g.H + 31) / 32, g.D * nbatch);
        transpose_flip_kernel<TI><<<tg, dim3(32, 8), 0, st>>>(in, volT, g.H, g.W, g.H);
        if (int rc = check_cuda("transpose")) return rc;
        const int nwarp = std::min(8, (g.Nv + CELL_R - 1) / CELL_R);
        const int rows_per_cta = nwarp * CELL_R;
        const int total = nview * nbatch;
        for (int z0 = 0; z0 < total; z0 += 65535) {
            const int nz = std::min(65535, total - z0);
            dim3 grid((g.Nu + 31) / 32, (g.Nv + rows_per_cta - 1) / rows_per_cta, nz);
            dim3 block(32, nwarp);
            if (eff == OP_A)
                cell_gather3d_kernel<TI, TO, CELL_R, OP_A><<<grid, block, 0, st>>>(g, vt, in, volT, out, nview, z0, z0dz, zd0, dvv, cw);
            else if (eff == OP_BT)
                cell_gather3d_kernel<TI, TO, CELL_R, OP_BT><<<grid, block, 0, st>>>(g, vt, in, volT, out, nview, z0, z0dz, zd0, dvv, cw);
            else
                cell_gather3d_kernel<TI, TO, CELL_R, OP_BWT><<<grid, block, 0, st>>>(g, vt, in, volT, out, nview, z0, z0dz, zd0, dvv, cw);
            if (int rc = check_cuda("cell_gather3d")) return rc;
        }
        return XR_OK;
    }
    // voxel gather
    const int nzg = (g.D + VOX_NW * VOX_R - 1) / (VOX_NW * VOX_R);
    if ((long long)nzg * nbatch > 65535) return fail(XR_ERR_UNSUPPORTED, "depth x batch too large for one launch");
    if (g.H > 65535) return fail(XR_ERR_UNSUPPORTED, "image height above 65535");
    dim3 grid((g.W + 31) / 32, g.H, nzg * nbatch);
    dim3 block(32, VOX_NW);
    const GeomF gf = make_geomf(g, 1);
    const float atconst = (float)(g.dx * g.dy * g.dz / (g.du * g.dv));
    // the prefix kernel addresses one view's table with 32-bit byte offsets
    const bool prefix_ok = (double)(g.Nv + 2) * g.Nu * sizeof(float2) < 2147483648.0;
    if (!g_force_plain && prefix_ok) {
        float2* tab = reinterpret_cast<float2*>(ws + l.sinoS);
        const int nbv = nbatch * nview;
        dim3 pg((g.Nu + 127) / 128, std::min(nbv, 65535));
        if (eff == OP_AT && g.type != GEO_PARALLEL)
            row_prefix3d_kernel<TI, true><<<pg, 128, 0, st>>>(g, vt, in, tab, nview, nbv, zd0, dvv);
        else
            row_prefix3d_kernel<TI, false><<<pg, 128, 0, st>>>(g, vt, in, tab, nview, nbv, zd0, dvv);
        if (int rc = check_cuda("row_prefix3d")) return rc;
        const int nzp = (g.D + PFX_R - 1) / PFX_R;
        if ((long long)nzp * nbatch > 65535) return fail(XR_ERR_UNSUPPORTED, "depth x batch too large for one launch");
        if (!(g_host_hooks & XR_HOOK_PFX_NOSTAGE)) {
            const int rc = run_pfx_stage<TO>(eff, g, gf, vt, tab, out, nbatch, nview, nzp, ws, l, st, z0dz, zd0, dvv,
                                             cw, atconst, oscale);
            if (rc >= 0) return rc;
        }
        dim3 pgrid((g.W + 31) / 32, (g.H + PFX_NWY - 1) / PFX_NWY, nzp * nbatch);
        dim3 pblock(32, PFX_NWY);
        if (eff == OP_AT)
            vox_prefix3d_kernel<TO, PFX_R, PFX_NWY, OP_AT><<<pgrid, pblock, 0, st>>>(
                g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, cw, atconst, oscale);
        else if (vt.arc && eff == OP_B)
            vox_prefix3d_kernel<TO, PFX_R, PFX_NWY, OP_B, false, true><<<pgrid, pblock, 0, st>>>(
                g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, cw, atconst, oscale);
        else if (vt.arc)
            vox_prefix3d_kernel<TO, PFX_R, PFX_NWY, OP_BW, false, true><<<pgrid, pblock, 0, st>>>(
                g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, cw, atconst, oscale);
        else if (eff == OP_B)
            vox_prefix3d_kernel<TO, PFX_R, PFX_NWY, OP_B><<<pgrid, pblock, 0, st>>>(
                g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, cw, atconst, oscale);
        else
            vox_prefix3d_kernel<TO, PFX_R, PFX_NWY, OP_BW><<<pgrid, pblock, 0, st>>>(
                g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, cw, atconst, oscale);
        return check_cuda("vox_prefix3d");
    }
    if (eff == OP_AT) {
        if (g.type != GEO_PARALLEL) {
            float* sinoS = reinterpret_cast<float*>(ws + l.sinoS);
            const size_t total = (size_t)nbatch * nview * g.Nv * g.Nu;
            prescale_at3d_kernel<TI><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(g, vt, in, sinoS, nview, total, zd0, dvv);
            if (int rc = check_cuda("prescale_at3d")) return rc;
            vox_gather3d_kernel<float, TO, VOX_R, OP_AT><<<grid, block, 0, st>>>(
                g, gf, vt, sinoS, out, nview, nzg, z0dz, zd0, dvv, cw, atconst, oscale);
        } else {
            vox_gather3d_kernel<TI, TO, VOX_R, OP_AT><<<grid, block, 0, st>>>(
                g, gf, vt, in, out, nview, nzg, z0dz, zd0, dvv, cw, atconst, oscale);
        }
    } else if (eff == OP_B) {
        vox_gather3d_kernel<TI, TO, VOX_R, OP_B><<<grid, block, 0, st>>>(
            g, gf, vt, in, out, nview, nzg, z0dz, zd0, dvv, cw, atconst, oscale);
    } else {
        vox_gather3d_kernel<TI, TO, VOX_R, OP_BW><<<grid, block, 0, st>>>(
            g, gf, vt, in, out, nview, nzg, z0dz, zd0, dvv, cw, atconst, oscale);
    }
    return check_cuda("vox_gather3d");
}

template <typename TI, typename TO>
int run2d(int op, const Geom& g, const TI* in, TO* out, const float* ang, int nbatch, int nview,
          char* ws, const Layout& l, cudaStream_t st, float oscale) {
    const ViewTables vt = tables_at(ws, l);
    const float cw = column_width(g, 0);
    if (nview == 0) {
        if (op == OP_AT || op == OP_B || op == OP_BW) {
            if (cudaMemsetAsync(out, 0, (size_t)g.H * g.W * nbatch * sizeof(TO), st) != cudaSuccess)
                return fail(XR_ERR_CUDA, "memset failed");
        }
        return XR_OK;
    }
    {
        dim3 grid((g.Nu + 1 + 127) / 128, nview);
        setup_views_kernel<<<grid, 128, 0, st>>>(g, 0, ang, nview, vt);
        if (int rc = check_cuda("setup_views")) return rc;
    }
    if (nview > 65535 || nbatch > 65535) return fail(XR_ERR_UNSUPPORTED, "views or batch above 65535");
    if (op == OP_A || op == OP_BT || op == OP_BWT) {
        TI* imgT = reinterpret_cast<TI*>(ws + l.volT);
        dim3 tg((g.W + 31) / 32, (g.H + 31) / 32, nbatch);
        transpose_flip_kernel<TI><<<tg, dim3(32, 8), 0, st>>>(in, imgT, g.H, g.W, g.H);
        if (int rc = check_cuda("transpose")) return rc;
        dim3 grid((g.Nu + 127) / 128, nview, nbatch);
        if (op == OP_A)
            cell_gather2d_kernel<TI, TO, OP_A><<<grid, 128, 0, st>>>(g, vt, in, imgT, out, nview, cw);
        else if (op == OP_BT)
            cell_gather2d_kernel<TI, TO, OP_BT><<<grid, 128, 0, st>>>(g, vt, in, imgT, out, nview, cw);
        else
            cell_gather2d_kernel<TI, TO, OP_BWT><<<grid, 128, 0, st>>>(g, vt, in, imgT, out, nview, cw);
        return check_cuda("cell_gather2d");
    }
    dim3 grid((g.W + 31) / 32, (g.H + 7) / 8, nbatch);
    dim3 block(32, 8);
    if (op == OP_AT)
        vox_gather2d_kernel<TI, TO, OP_AT><<<grid, block, 0, st>>>(g, vt, in, out, nview, cw, oscale);
    else if (op == OP_B)
        vox_gather2d_kernel<TI, TO, OP_B><<<grid, block, 0, st>>>(g, vt, in, out, nview, cw, oscale);
    else
        vox_gather2d_kernel<TI, TO, OP_BW><<<grid, block, 0, st>>>(g, vt, in, out, nview, cw, oscale);
    return check_cuda("vox_gather2d");
}

template <typename TI>
int dispatch_out(int dim3d, int op, const Geom& g, const void* in, void* out, int dto, const float* ang,
                 int nbatch, int nview, char* ws, const Layout& l, cudaStream_t st, float oscale) {
    const TI* i = static_cast<const TI*>(in);
    if (dto == DT_F32) {
        float* o = static_cast<float*>(out);
        return dim3d ? run3d(op, g, i, o, ang, nbatch, nview, ws, l, st, oscale)
                     : run2d(op, g, i, o, ang, nbatch, nview, ws, l, st, oscale);
    }
    if (dto == DT_BF16) {
        __nv_bfloat16* o = static_cast<__nv_bfloat16*>(out);
        return dim3d ? run3d(op, g, i, o, ang, nbatch, nview, ws, l, st, oscale)
                     : run2d(op, g, i, o, ang, nbatch, nview, ws, l, st, oscale);
    }
    __half* o = static_cast<__half*>(out);
    return dim3d ? run3d(op, g, i, o, ang, nbatch, nview, ws, l, st, oscale)
                 : run2d(op, g, i, o, ang, nbatch, nview, ws, l, st, oscale);
}

int apply(int dim3d, int op, const Geom& g, const void* in, int dti, void* out, int dto, const float* ang,
          int nbatch, int nview, void* workspace, size_t ws_bytes, void* stream, float oscale) {
    if (int rc = validate(g, dim3d, op, nbatch, nview)) return rc;
    if (!dtype_ok(dti) || !dtype_ok(dto)) return fail(XR_ERR_INVALID_ARGUMENT, "unsupported dtype (%d, %d)", dti, dto);
    // With zero views the sinogram side is empty and may be a null pointer.
    const bool sino_in = (op == OP_AT || op == OP_B || op == OP_BW);
    if ((!in && !(sino_in && nview == 0)) || (!out && !(!sino_in && nview == 0)))
        return fail(XR_ERR_INVALID_ARGUMENT, "null input or output pointer");
    if (nview > 0 && !ang) return fail(XR_ERR_INVALID_ARGUMENT, "null angles pointer");
    const Layout l = layout(dim3d, op, g, nbatch, nview, dti);
    if (!workspace || ws_bytes < l.total)
        return fail(XR_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", l.total, ws_bytes);
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
        return fail(XR_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    if (dti == DT_F32) return dispatch_out<float>(dim3d, op, g, in, out, dto, ang, nbatch, nview, ws, l, st, oscale);
    if (dti == DT_BF16) return dispatch_out<__nv_bfloat16>(dim3d, op, g, in, out, dto, ang, nbatch, nview, ws, l, st, oscale);
    return dispatch_out<__half>(dim3d, op, g, in, out, dto, ang, nbatch, nview, ws, l, st, oscale);
}

// ------------------------------------------------------ system matrix export

// Layout of the per-view tables alone (no operator-specific regions).
Layout tables_layout(int dim3d, const Geom& g, int nview) { return layout(dim3d, -1, g, 1, nview, DT_F32); }

int sysmat(int dim3d, const Geom& g, const float* ang, int nview, const long long* offsets, long long* counts,
           long long* rows, long long* cols, float* vals, void* workspace, size_t ws_bytes, void* stream) {
    if (int rc = validate(g, dim3d, OP_A, 1, nview)) return rc;
    if (nview < 1 || !ang) return fail(XR_ERR_INVALID_ARGUMENT, "need at least one view and its angle");
    if (!offsets && !counts) return fail(XR_ERR_INVALID_ARGUMENT, "count pass needs the counts buffer");
    if (offsets && (!rows || !cols || !vals)) return fail(XR_ERR_INVALID_ARGUMENT, "fill pass needs rows, cols, vals");
    const Layout l = tables_layout(dim3d, g, nview);
    if (!workspace || ws_bytes < l.total)
        return fail(XR_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", l.total, ws_bytes);
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
        return fail(XR_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const ViewTables vt = tables_at(static_cast<char*>(workspace), l);
    {
        dim3 grid((g.Nu + 1 + 127) / 128, nview);
        setup_views_kernel<<<grid, 128, 0, st>>>(g, dim3d, ang, nview, vt);
        if (int rc = check_cuda("setup_views")) return rc;
    }
    double zd0 = 0.0, dvv = 1.0, z0dz = 0.0;
    if (dim3d) row_params(g, zd0, dvv, z0dz);
    const long long ncell = (long long)nview * (dim3d ? g.Nv : 1) * g.Nu;
    const unsigned blocks = (unsigned)((ncell + 127) / 128);
    if (dim3d) {
        if (offsets) sysmat_kernel<true, true><<<blocks, 128, 0, st>>>(g, vt, nview, counts, offsets, rows, cols, vals, z0dz, zd0, dvv);
        else sysmat_kernel<false, true><<<blocks, 128, 0, st>>>(g, vt, nview, counts, offsets, rows, cols, vals, z0dz, zd0, dvv);
    } else {
        if (offsets) sysmat_kernel<true, false><<<blocks, 128, 0, st>>>(g, vt, nview, counts, offsets, rows, cols, vals, z0dz, zd0, dvv);
        else sysmat_kernel<false, false><<<blocks, 128, 0, st>>>(g, vt, nview, counts, offsets, rows, cols, vals, z0dz, zd0, dvv);
    }
    return check_cuda("sysmat");
}

// ------------------------------------------------------ helical scans

struct HelLayout {
    Layout l;  // view tables (+ the flipped image for A / B^T, row prefix tables for B, A^T, Bw)
    size_t hel, wv, zw, scan, wtab, scale, imgs, imgsT, total;
};

HelLayout hel_layout(int op, const Geom& g, int nbatch, int nview) {
    HelLayout h;
    h.l = layout(1, op, g, nbatch, nview, DT_F32, false);
    size_t o = h.l.total;
    const size_t V = (size_t)(nview > 0 ? nview : 1);
    h.hel = o;  o = align256(o + V * sizeof(HelView));
    h.wv = o;   o = align256(o + V * sizeof(HelWView));
    h.zw = h.scan = h.wtab = h.scale = h.imgs = h.imgsT = o;
    if (op == OP_BW || op == OP_BWT) {
        const size_t nvox = (size_t)g.D * g.H * g.W;
        h.zw = o;    o = align256(o + (size_t)g.D * sizeof(HelZ));
        h.scan = o;  o = align256(o + sizeof(HelScanF));
        h.wtab = o;  o = align256(o + (size_t)(g.D + 3) * V * sizeof(float));  // slices -1 .. D + 1
        if (op == OP_BWT) {
            h.scale = o; o = align256(o + nvox * sizeof(float));
            h.imgs = o;  o = align256(o + (size_t)nbatch * nvox * sizeof(float));
            h.imgsT = o; o = align256(o + (size_t)nbatch * nvox * sizeof(float));
        }
    }
    h.total = o;
    return h;
}

constexpr int HEL_WBP_R = 8;
constexpr int HEL_WBP_NWY = 8;
constexpr int HEL_WBPT_R = 8;

int helical(int op, const Geom& g, const HelOpts& o, const float* in, float* out, const float* ang,
            const float* sp, int nbatch, int nview, void* workspace, size_t ws_bytes, void* stream) {
    if (int rc = validate(g, 1, op, nbatch, nview)) return rc;
    if (g.type != GEO_ARC)
        return fail(XR_ERR_INVALID_ARGUMENT, "helical operators need the arc detector (type 2), got %d", g.type);
    if (nview < 1) return fail(XR_ERR_INVALID_ARGUMENT, "helical operators need at least one view");
    if (!in || !out || !ang || !sp) return fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    if (o.view_mode < 0 || o.view_mode > 3) return fail(XR_ERR_INVALID_ARGUMENT, "view mode %d not in 0..3", o.view_mode);
    if (o.weight_mode < 0 || o.weight_mode > 1)
        return fail(XR_ERR_INVALID_ARGUMENT, "weight mode %d not in 0..1", o.weight_mode);
    const HelLayout hl = hel_layout(op, g, nbatch, nview);
    if (!workspace || ws_bytes < hl.total)
        return fail(XR_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", hl.total, ws_bytes);
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
        return fail(XR_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    ViewTables vt = tables_at(ws, hl.l);
    vt.hel = reinterpret_cast<HelView*>(ws + hl.hel);
    HelWView* wv = reinterpret_cast<HelWView*>(ws + hl.wv);
    {
        dim3 grid((g.Nu + 1 + 127) / 128, nview);
        setup_views_helical_kernel<<<grid, 128, 0, st>>>(g, ang, sp, nview, vt, wv);
        if (int rc = check_cuda("setup_views_helical")) return rc;
    }
    double zd0, dvv, z0dz;
    row_params(g, zd0, dvv, z0dz);  // dvv; the z placement is per view
    const GeomF gf = make_geomf(g, 1);
    if (op == OP_A || op == OP_BT) {
        if (!g_force_plain) {
            const int rc = run_cell_tma<float, float, true>(op, g, in, out, nbatch, nview, ws, hl.l, vt, st, z0dz,
                                                              zd0, dvv, 0.0f);
            if (rc >= 0) return rc;
        }
        float* volT = reinterpret_cast<float*>(ws + hl.l.volT);
        dim3 tg((g.W + 31) / 32, (g.H + 31) / 32, g.D * nbatch);
        transpose_flip_kernel<float><<<tg, dim3(32, 8), 0, st>>>(in, volT, g.H, g.W, g.H);
        if (int rc = check_cuda("transpose")) return rc;
        const int nwarp = std::min(8, (g.Nv + CELL_R - 1) / CELL_R);
        const int rows_per_cta = nwarp * CELL_R;
        const int total = nview * nbatch;
        for (int v0 = 0; v0 < total; v0 += 65535) {
            const int nz = std::min(65535, total - v0);
            dim3 grid((g.Nu + 31) / 32, (g.Nv + rows_per_cta - 1) / rows_per_cta, nz);
            if (op == OP_A)
                cell_gather3d_kernel<float, float, CELL_R, OP_A, true><<<grid, dim3(32, nwarp), 0, st>>>(
                    g, vt, in, volT, out, nview, v0, z0dz, zd0, dvv, 0.0f);
            else
                cell_gather3d_kernel<float, float, CELL_R, OP_BT, true><<<grid, dim3(32, nwarp), 0, st>>>(
                    g, vt, in, volT, out, nview, v0, z0dz, zd0, dvv, 0.0f);
            if (int rc = check_cuda("cell_gather3d")) return rc;
        }
        return XR_OK;
    }
    if ((double)(g.Nv + 2) * g.Nu * sizeof(float2) >= 2147483648.0)
        return fail(XR_ERR_UNSUPPORTED, "detector of %d x %d cells too large for one view's row table", g.Nu, g.Nv);
    HelZ* zw = reinterpret_cast<HelZ*>(ws + hl.zw);
    HelScanF* scan = reinterpret_cast<HelScanF*>(ws + hl.scan);
    float* wtab_pad = reinterpret_cast<float*>(ws + hl.wtab);  // slice j at row j + 1
    float* wtab = wtab_pad + nview;                             // slice j at row j
    float* scale = reinterpret_cast<float*>(ws + hl.scale);
    const int nzg = (g.D + HEL_WBP_R - 1) / HEL_WBP_R;
    if (op == OP_BW || op == OP_BWT) {
        if ((long long)nzg * nbatch > 65535) return fail(XR_ERR_UNSUPPORTED, "depth x batch too large for one launch");
        hel_zwin_kernel<<<(g.D + 127) / 128, 128, 0, st>>>(g, o, ang, sp, nview, zw, scan);
        if (int rc = check_cuda("hel_zwin")) return rc;
        hel_wtab_kernel<<<dim3((nview + 127) / 128, g.D + 3), 128, 0, st>>>(scan, wv, zw, g.D, nview, wtab_pad);
        if (int rc = check_cuda("hel_wtab")) return rc;
    }
    if (op == OP_BWT) {
        dim3 grid((g.W + 31) / 32, (g.H + HEL_WBP_NWY - 1) / HEL_WBP_NWY, nzg);
        hel_wbp_kernel<HEL_WBP_R, HEL_WBP_NWY, false><<<grid, dim3(32, HEL_WBP_NWY), 0, st>>>(
            g, gf, vt, o, scan, wv, zw, wtab, ang, sp, nullptr, scale, nview, nzg, dvv);
        if (int rc = check_cuda("hel_wbp (normalisation)")) return rc;
        float* imgs = reinterpret_cast<float*>(ws + hl.imgs);
        const size_t nvox = (size_t)g.D * g.H * g.W, n = nvox * nbatch;
        hel_prescale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, scale, imgs, nvox, n);
        if (int rc = check_cuda("hel_prescale")) return rc;
        // The tabulated slices through the TMA cell gather (their weight is
        // one number per slice and view); the others, if any, added by the
        // per-voxel gather.  Without a TMA plan the per-voxel gather does all.
        int rc_tma = -1;
        if (!g_force_plain) {
            rc_tma = run_cell_tma<float, float, true>(OP_BWT, g, imgs, out, nbatch, nview, ws, hl.l, vt, st, z0dz,
                                                      zd0, dvv, (float)g.sod * (float)g.du, wtab_pad);
            if (rc_tma > 0) return rc_tma;
        }
        float* imgsT = reinterpret_cast<float*>(ws + hl.imgsT);
        dim3 tg((g.W + 31) / 32, (g.H + 31) / 32, g.D * nbatch);
        transpose_flip_kernel<float><<<tg, dim3(32, 8), 0, st>>>(imgs, imgsT, g.H, g.W, g.H);
        if (int rc = check_cuda("transpose")) return rc;
        const int nwarp = std::min(8, (g.Nv + HEL_WBPT_R - 1) / HEL_WBPT_R);
        const int rows_per_cta = nwarp * HEL_WBPT_R;
        const int total = nview * nbatch;
        for (int v0 = 0; v0 < total; v0 += 65535) {
            const int nz = std::min(65535, total - v0);
            dim3 grid((g.Nu + 31) / 32, (g.Nv + rows_per_cta - 1) / rows_per_cta, nz);
            if (rc_tma == 0)
                hel_wbpt_kernel<HEL_WBPT_R, true><<<grid, dim3(32, nwarp), 0, st>>>(
                    g, vt, o, scan, wv, zw, wtab, ang, sp, imgs, imgsT, out, nview, v0, dvv);
            else
                hel_wbpt_kernel<HEL_WBPT_R, false><<<grid, dim3(32, nwarp), 0, st>>>(
                    g, vt, o, scan, wv, zw, wtab, ang, sp, imgs, imgsT, out, nview, v0, dvv);
            if (int rc = check_cuda("hel_wbpt")) return rc;
        }
        return XR_OK;
    }
    float2* tab = reinterpret_cast<float2*>(ws + hl.l.sinoS);
    const int nbv = nbatch * nview;
    dim3 pg((g.Nu + 127) / 128, std::min(nbv, 65535));
    if (op == OP_AT)
        row_prefix3d_kernel<float, true, true><<<pg, 128, 0, st>>>(g, vt, in, tab, nview, nbv, zd0, dvv);
    else
        row_prefix3d_kernel<float, false><<<pg, 128, 0, st>>>(g, vt, in, tab, nview, nbv, zd0, dvv);
    if (int rc = check_cuda("row_prefix3d")) return rc;
    if (op == OP_BW) {
        dim3 grid((g.W + 31) / 32, (g.H + HEL_WBP_NWY - 1) / HEL_WBP_NWY, nzg * nbatch);
        hel_wbp_kernel<HEL_WBP_R, HEL_WBP_NWY, true><<<grid, dim3(32, HEL_WBP_NWY), 0, st>>>(
            g, gf, vt, o, scan, wv, zw, wtab, ang, sp, tab, out, nview, nzg, dvv);
        return check_cuda("hel_wbp");
    }
    const int nzp = (g.D + PFX_R - 1) / PFX_R;
    if ((long long)nzp * nbatch > 65535) return fail(XR_ERR_UNSUPPORTED, "depth x batch too large for one launch");
    dim3 pgrid((g.W + 31) / 32, (g.H + PFX_NWY - 1) / PFX_NWY, nzp * nbatch);
    dim3 pblock(32, PFX_NWY);
    const float atconst = (float)(g.dx * g.dy * g.dz / (g.du * g.dv));
    // the table footprints staged in shared memory (the box from the plan of
    // the same volume and detector on a circular scan; views whose box does
    // not fit go to the fallback launch)
    if (!(g_host_hooks & XR_HOOK_PFX_NOSTAGE)) {
        const int rc = run_pfx_stage<float, true>(op, g, gf, vt, tab, out, nbatch, nview, nzp, ws, hl.l, st, z0dz, zd0,
                                                  dvv, 0.0f, atconst, 1.0f);
        if (rc >= 0) return rc;
    }
    if (op == OP_AT)
        vox_prefix3d_kernel<float, PFX_R, PFX_NWY, OP_AT, true><<<pgrid, pblock, 0, st>>>(
            g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, 0.0f, atconst, 1.0f);
    else
        vox_prefix3d_kernel<float, PFX_R, PFX_NWY, OP_B, true><<<pgrid, pblock, 0, st>>>(
            g, gf, vt, tab, out, nview, nzp, z0dz, zd0, dvv, 0.0f, atconst, 1.0f);
    return check_cuda("vox_prefix3d");
}

// ------------------------------------------------------ ragged 2D batches

struct RaggedLayout {
    size_t desc, sync;
    std::vector<size_t> hdr, bA, bB, colQ, colR, colE, colF, colM, arc, imgT, filt;
    size_t total;
};

}  // namespace
}  // namespace xr

struct xr_ragged2d_plan {
    std::vector<xr_ragged2d_instance> inst;
    std::vector<xr::Geom> geom;
    xr::RaggedLayout lay;
    int t0[10][1];  // unused placeholder (tile starts live in the device descriptors)
    std::vector<std::array<int, 10>> starts;  // per instance
    int totals[10];
    int max_nu;
    int device;
    int grid;
    size_t smem;
    void* workspace;
};

namespace xr {
namespace {

int ragged_tiles(const Geom& g, int nview, int list) {
    const int hw = g.H * g.W;
    if (list == 0) return nview + (hw + 1023) / 1024;
    if (list == 1) return nview;
    if (list < 6) return nview * ((g.Nu + (32 << (list - 2)) - 1) / (32 << (list - 2)));
    const int px = 256 / (1 << (list - 6));
    return (hw + px - 1) / px;
}

// Fixed device scratch of xr_dd2d_noalloc, the entry for callers that cannot
// allocate device memory mid-run.  Host code only sees a stand-in for this
// name, so its device address is looked up once per device, with that
// device current (cudaGetSymbolAddress), cached, and passed to the kernels;
// nothing is ever allocated for it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[XR_NOALLOC_SCRATCH_BYTES];

// The address is cached per device and per context: after a device reset
// the primary context (and the module holding the array) is created anew, and
// the array gets a new address.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);

int noalloc_scratch(void** ptr) {
    static std::mutex mu;
    static std::vector<std::pair<CUcontext, void*>> by_device;
    static CtxGetCurrentFn ctx_current = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(XR_ERR_CUDA, "cudaGetDevice failed");
    std::lock_guard<std::mutex> lock(mu);
    if (!ctx_current) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return fail(XR_ERR_CUDA, "cuCtxGetCurrent is not available");
        ctx_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    if ((int)by_device.size() <= dev) by_device.resize(dev + 1, {nullptr, nullptr});
    CUcontext ctx = nullptr;
    if (ctx_current(&ctx) == CUDA_SUCCESS && ctx && by_device[dev].first == ctx && by_device[dev].second) {
        *ptr = by_device[dev].second;
        return XR_OK;
    }
    // first call on this device or context (the lookup creates the primary
    // context when there is none yet)
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(XR_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
    if (ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return fail(XR_ERR_CUDA, "no current CUDA context");
    by_device[dev] = {ctx, p};
    *ptr = p;
    return XR_OK;
}

}  // namespace

// NVTX range over one C-ABI call: host markers for a profiler's timeline
// (nvtx3 is header-only and does next to nothing when no tool is attached).
struct Trace {
    explicit Trace(const char* name) { nvtxRangePushA(name); }
    ~Trace() { nvtxRangePop(); }
    Trace(const Trace&) = delete;
    Trace& operator=(const Trace&) = delete;
};

// "<entry> <operator>" for the range names of the DD entry points
inline const char* op_trace_name(int dim, int op) {
    static const char* const names[3][6] = {
        {"xr_dd2d A", "xr_dd2d AT", "xr_dd2d B", "xr_dd2d BT", "xr_dd2d BW", "xr_dd2d BWT"},
        {"xr_dd3d A", "xr_dd3d AT", "xr_dd3d B", "xr_dd3d BT", "xr_dd3d BW", "xr_dd3d BWT"},
        {"xr_helical3d A", "xr_helical3d AT", "xr_helical3d B", "xr_helical3d BT", "xr_helical3d BW",
         "xr_helical3d BWT"}};
    static const char* const other[3] = {"xr_dd2d", "xr_dd3d", "xr_helical3d"};
    return (op >= 0 && op < 6) ? names[dim][op] : other[dim];
}

// FFT filter (xr_fft_filter.cuh) of `nrows` rows from `rows_src`: one wave of
// CTAs, each transforming the filter once and then a share of the rows.
template <typename RowsT>
int launch_fft_filter(const RowsT& rows_src, float* out, int nrows, int Nu, const float* filt, cudaStream_t st) {
    const int m = fft_log2_for(Nu);
    const size_t smem = fft_filter_smem(m);
    auto k = fft_filter_kernel<RowsT>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(XR_ERR_CUDA, "cannot reserve %zu bytes of shared memory", smem);
    int dev = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, XR_FFT_THREADS, smem) != cudaSuccess || per_sm < 1)
        return fail(XR_ERR_CUDA, "cannot size the FFT filter grid");
    const int nquad = (nrows + 3) / 4;  // four rows per CTA iteration
    const int grid = std::min(nquad, per_sm * nsm);
    k<<<grid, XR_FFT_THREADS, smem, st>>>(rows_src, out, nrows, Nu, filt, m);
    return XR_OK;
}

}  // namespace xr

extern "C" {

size_t xr_dd2d_workspace_size(int op, const xr_geom2d* geom, int nbatch, int nview) {
    if (!geom) return 0;
    const xr::Geom g = xr::geom_from(geom);
    return xr::layout(0, op, g, nbatch, nview, xr::DT_F32).total;
}

size_t xr_dd3d_workspace_size(int op, const xr_geom3d* geom, int nbatch, int nview) {
    if (!geom) return 0;
    const xr::Geom g = xr::geom_from(geom);
    // enough for every storage type (half-precision images add a widened copy)
    return std::max(xr::layout(1, op, g, nbatch, nview, xr::DT_F32).total,
                    xr::layout(1, op, g, nbatch, nview, xr::DT_BF16).total);
}

int xr_dd2d(int op, const xr_geom2d* geom, const void* in, int dtype_in, void* out, int dtype_out,
            const float* angles, int nbatch, int nview, void* workspace, size_t workspace_bytes,
            void* stream) {
    xr::Trace tr(xr::op_trace_name(0, op));
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    return xr::apply(0, op, xr::geom_from(geom), in, dtype_in, out, dtype_out, angles, nbatch, nview,
                     workspace, workspace_bytes, stream, 1.0f);
}

int xr_dd3d(int op, const xr_geom3d* geom, const void* in, int dtype_in, void* out, int dtype_out,
            const float* angles, int nbatch, int nview, void* workspace, size_t workspace_bytes,
            void* stream) {
    xr::Trace tr(xr::op_trace_name(1, op));
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    return xr::apply(1, op, xr::geom_from(geom), in, dtype_in, out, dtype_out, angles, nbatch, nview,
                     workspace, workspace_bytes, stream, 1.0f);
}

size_t xr_helical3d_workspace_size(int op, const xr_geom3d* geom, int nbatch, int nview) {
    if (!geom) return 0;
    return xr::hel_layout(op, xr::geom_from(geom), nbatch, nview).total;
}

int xr_helical3d(int op, const xr_geom3d* geom, const xr_helical_opts* opts, const float* in, float* out,
                 const float* angles, const float* source_pos, int nbatch, int nview, void* workspace,
                 size_t workspace_bytes, void* stream) {
    xr::Trace tr(xr::op_trace_name(2, op));
    if (!geom || !opts) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry or options");
    xr::HelOpts o;
    o.view_mode = opts->view_mode;
    o.weight_mode = opts->weight_mode;
    o.view_turns = opts->view_turns;
    o.halfscan_coef = opts->halfscan_coef;
    o.tang_k = opts->tang_k;
    o.tang_blend = opts->tang_blend;
    return xr::helical(op, xr::geom_from(geom), o, in, out, angles, source_pos, nbatch, nview, workspace,
                       workspace_bytes, stream);
}

int xr_fbp_filter(const void* in, int dtype_in, float* out, int nrows, int Nu, int nview, int rows_per_view,
                  const float* cosw, const float* filt, const float* parker, void* stream) {
    xr::Trace tr("xr_fbp_filter");
    if (!in || !out || !filt) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    if (Nu < 1 || nrows < 0 || nview < 1 || rows_per_view < 1)
        return xr::fail(XR_ERR_INVALID_ARGUMENT, "bad filter sizes");
    if (nrows == 0) return XR_OK;
    if (!xr::dtype_ok(dtype_in)) return xr::fail(XR_ERR_INVALID_ARGUMENT, "unsupported dtype %d", dtype_in);
    if (!xr::g_force_plain && xr::fft_log2_for(Nu) <= xr::XR_FFT_MAX_LOG) {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        int rc;
        if (dtype_in == xr::DT_F32)
            rc = xr::launch_fft_filter(xr::SinoRows<float>{static_cast<const float*>(in), cosw, parker, Nu, nview, rows_per_view}, out, nrows, Nu, filt, st);
        else if (dtype_in == xr::DT_BF16)
            rc = xr::launch_fft_filter(xr::SinoRows<__nv_bfloat16>{static_cast<const __nv_bfloat16*>(in), cosw, parker, Nu, nview, rows_per_view}, out, nrows, Nu, filt, st);
        else
            rc = xr::launch_fft_filter(xr::SinoRows<__half>{static_cast<const __half*>(in), cosw, parker, Nu, nview, rows_per_view}, out, nrows, Nu, filt, st);
        if (rc) return rc;
        return xr::check_cuda("fft_filter");
    }
    constexpr int OUTS = 8;
    // threads per row (a warp multiple covering Nu / 8 outputs), rows per CTA
    const int tpr = std::min(256, ((Nu + OUTS - 1) / OUTS + 31) / 32 * 32);
    const int rpc = std::max(1, 256 / tpr);
    const size_t smem = ((size_t)(xr::filt_taps_smem(Nu) + 3) / 4 * 4 + (size_t)rpc * xr::filt_row_pitch(Nu)) * sizeof(float);
    if (smem > 200 * 1024) return xr::fail(XR_ERR_UNSUPPORTED, "detector width %d too large for the filter kernel", Nu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = std::min((nrows + rpc - 1) / rpc, 148 * 8);
    auto launch = [&](auto rows_src) -> int {
        auto k = xr::fbp_filter_kernel<decltype(rows_src), OUTS>;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return xr::fail(XR_ERR_CUDA, "cannot reserve %zu bytes of shared memory", smem);
        k<<<grid, 256, smem, st>>>(rows_src, out, nrows, Nu, filt, tpr, rpc);
        return XR_OK;
    };
    int rc;
    if (dtype_in == xr::DT_F32)
        rc = launch(xr::SinoRows<float>{static_cast<const float*>(in), cosw, parker, Nu, nview, rows_per_view});
    else if (dtype_in == xr::DT_BF16)
        rc = launch(xr::SinoRows<__nv_bfloat16>{static_cast<const __nv_bfloat16*>(in), cosw, parker, Nu, nview, rows_per_view});
    else
        rc = launch(xr::SinoRows<__half>{static_cast<const __half*>(in), cosw, parker, Nu, nview, rows_per_view});
    if (rc) return rc;
    return xr::check_cuda("fbp_filter");
}

const char* xr_last_error(void) { return xr::g_last_error.c_str(); }

int xr_cell_plan(const xr_geom3d* geom, int* ok, int* box_pixels, int* box_z, int* rows_per_thread, int* fine) {
    if (!geom || !ok || !box_pixels || !box_z || !rows_per_thread || !fine)
        return xr::fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    const xr::Geom g = xr::geom_from(geom);
    if (int rc = xr::validate(g, 1, 0, 1, 1)) return rc;
    const xr::CellPlan p = xr::plan_cell(g);
    *ok = p.ok;
    *box_pixels = p.BP;
    *box_z = p.BZ;
    *rows_per_thread = p.R;
    *fine = p.fine;
    return XR_OK;
}

int xr_pfx_stage_plan(const xr_geom3d* geom, int* ok, int* box_cols, int* box_rows) {
    if (!geom || !ok || !box_cols || !box_rows) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    const xr::Geom g = xr::geom_from(geom);
    if (int rc = xr::validate(g, 1, 0, 1, 1)) return rc;
    const xr::PfxStagePlan p = xr::plan_pfx_stage(g);
    *ok = p.ok;
    *box_cols = p.BC;
    *box_rows = p.BR;
    return XR_OK;
}

int xr_set_plain_kernels(int on) {
    xr::g_force_plain = (on != 0);
    return XR_OK;
}

int xr_device_error(unsigned int* code, int clear) {
    if (!code) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    if (cudaMemcpyFromSymbol(code, xr::g_device_error, sizeof(unsigned int)) != cudaSuccess)
        return xr::fail(XR_ERR_CUDA, "reading the device error word failed");
    if (clear) {
        const unsigned int zero = 0;
        if (cudaMemcpyToSymbol(xr::g_device_error, &zero, sizeof(unsigned int)) != cudaSuccess)
            return xr::fail(XR_ERR_CUDA, "clearing the device error word failed");
    }
    return XR_OK;
}

int xr_set_wait_limits(long long tma_polls, long long barrier_polls) {
    const long long t = tma_polls > 0 ? tma_polls : xr::XR_WAIT_LIMIT_DEFAULT;
    const long long b = barrier_polls > 0 ? barrier_polls : xr::XR_BARRIER_LIMIT_DEFAULT;
    if (cudaMemcpyToSymbol(xr::g_wait_limit, &t, sizeof(t)) != cudaSuccess ||
        cudaMemcpyToSymbol(xr::g_barrier_limit, &b, sizeof(b)) != cudaSuccess)
        return xr::fail(XR_ERR_CUDA, "setting the wait limits failed");
    return XR_OK;
}

int xr_test_hooks(unsigned int hooks) {
    xr::g_host_hooks = hooks;
    if (cudaMemcpyToSymbol(xr::g_test_hooks, &hooks, sizeof(hooks)) != cudaSuccess)
        return xr::fail(XR_ERR_CUDA, "setting the test hooks failed");
    return XR_OK;
}

int xr_dd2d_noalloc(int op, const xr_geom2d* geom, const void* in, int dtype_in, void* out, int dtype_out,
                    const float* angles, int nbatch, int nview, void* stream) {
    xr::Trace tr("xr_dd2d_noalloc");
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    const xr::Geom g = xr::geom_from(geom);
    if (int rc = xr::validate(g, 0, op, nbatch, nview)) return rc;
    if (!xr::dtype_ok(dtype_in) || !xr::dtype_ok(dtype_out))
        return xr::fail(XR_ERR_INVALID_ARGUMENT, "unsupported dtype (%d, %d)", dtype_in, dtype_out);
    const size_t need = xr::layout(0, op, g, nbatch, nview, dtype_in).total;
    if (need > (size_t)XR_NOALLOC_SCRATCH_BYTES)
        return xr::fail(XR_ERR_WORKSPACE,
                        "request needs %zu bytes of scratch; xr_dd2d_noalloc has a fixed %zu-byte scratch "
                        "(use xr_dd2d with a caller workspace)",
                        need, (size_t)XR_NOALLOC_SCRATCH_BYTES);
    void* scratch = nullptr;
    if (int rc = xr::noalloc_scratch(&scratch)) return rc;
    return xr::apply(0, op, g, in, dtype_in, out, dtype_out, angles, nbatch, nview, scratch,
                     (size_t)XR_NOALLOC_SCRATCH_BYTES, stream, 1.0f);
}

unsigned long long xr_launch_count(void) { return xr::g_launches.load(std::memory_order_relaxed); }

int xr_rebin_parallel(const void* in, int dtype_in, float* out, int nbatch, int nview, int Nv, int Nu,
                      const float* grid, int nview_out, int Nt, const float* filt, void* stream) {
    using namespace xr;
    Trace tr("xr_rebin_parallel");
    if (!in || !out || !grid) return fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    if (nbatch < 0 || nview < 1 || Nv < 1 || Nu < 1 || nview_out < 0 || Nt < 1)
        return fail(XR_ERR_INVALID_ARGUMENT, "bad rebinning sizes");
    if (!dtype_ok(dtype_in)) return fail(XR_ERR_INVALID_ARGUMENT, "unsupported dtype %d", dtype_in);
    if (reinterpret_cast<uintptr_t>(grid) % 8 != 0) return fail(XR_ERR_INVALID_ARGUMENT, "grid must be 8-byte aligned");
    const long long total = (long long)nbatch * nview_out * Nv * Nt;
    if (total == 0) return XR_OK;
    if ((long long)nbatch * nview_out * Nv > 0x7fffffffll) return fail(XR_ERR_UNSUPPORTED, "too many rows");
    const RebinGrid r{grid, nview, Nv, Nu, nview_out, Nt};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!filt) {
        if (Nv > 65535) return fail(XR_ERR_UNSUPPORTED, "more than 65535 detector rows");
        const int nz = nbatch * nview_out;
        for (int z0 = 0; z0 < nz; z0 += 65535) {
            const dim3 grid((Nt + 255) / 256, Nv, std::min(65535, nz - z0));
            if (dtype_in == DT_F32) rebin_kernel<float><<<grid, 256, 0, st>>>(static_cast<const float*>(in), out, r, z0);
            else if (dtype_in == DT_BF16) rebin_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(in), out, r, z0);
            else rebin_kernel<__half><<<grid, 256, 0, st>>>(static_cast<const __half*>(in), out, r, z0);
            if (int rc = check_cuda("rebin")) return rc;
        }
        return XR_OK;
    }
    // rebinning fused into the filter kernel's row loads
    constexpr int OUTS = 8;
    const int nrows = (int)((long long)nbatch * nview_out * Nv);
    if (!g_force_plain && fft_log2_for(Nt) <= XR_FFT_MAX_LOG) {
        int rc;
        if (dtype_in == DT_F32) rc = launch_fft_filter(RebinRows<float>{static_cast<const float*>(in), r}, out, nrows, Nt, filt, st);
        else if (dtype_in == DT_BF16) rc = launch_fft_filter(RebinRows<__nv_bfloat16>{static_cast<const __nv_bfloat16*>(in), r}, out, nrows, Nt, filt, st);
        else rc = launch_fft_filter(RebinRows<__half>{static_cast<const __half*>(in), r}, out, nrows, Nt, filt, st);
        if (rc) return rc;
        return check_cuda("rebin_fft_filter");
    }
    const int tpr = std::min(256, ((Nt + OUTS - 1) / OUTS + 31) / 32 * 32);
    const int rpc = std::max(1, 256 / tpr);
    const size_t smem = ((size_t)(filt_taps_smem(Nt) + 3) / 4 * 4 + (size_t)rpc * filt_row_pitch(Nt)) * sizeof(float);
    if (smem > 200 * 1024) return fail(XR_ERR_UNSUPPORTED, "detector width %d too large for the filter kernel", Nt);
    const int grid_blocks = std::min((nrows + rpc - 1) / rpc, 148 * 8);
    auto launch = [&](auto rows_src) -> int {
        auto k = fbp_filter_kernel<decltype(rows_src), OUTS>;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return fail(XR_ERR_CUDA, "cannot reserve %zu bytes of shared memory", smem);
        k<<<grid_blocks, 256, smem, st>>>(rows_src, out, nrows, Nt, filt, tpr, rpc);
        return XR_OK;
    };
    int rc;
    if (dtype_in == DT_F32) rc = launch(RebinRows<float>{static_cast<const float*>(in), r});
    else if (dtype_in == DT_BF16) rc = launch(RebinRows<__nv_bfloat16>{static_cast<const __nv_bfloat16*>(in), r});
    else rc = launch(RebinRows<__half>{static_cast<const __half*>(in), r});
    if (rc) return rc;
    return check_cuda("rebin_filter");
}

size_t xr_sysmat2d_workspace_size(const xr_geom2d* geom, int nview) {
    if (!geom) return 0;
    return xr::tables_layout(0, xr::geom_from(geom), nview).total;
}

size_t xr_sysmat3d_workspace_size(const xr_geom3d* geom, int nview) {
    if (!geom) return 0;
    return xr::tables_layout(1, xr::geom_from(geom), nview).total;
}

int xr_sysmat2d(const xr_geom2d* geom, const float* angles, int nview, const long long* offsets, long long* counts,
                long long* rows, long long* cols, float* vals, void* workspace, size_t workspace_bytes, void* stream) {
    xr::Trace tr("xr_sysmat2d");
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    return xr::sysmat(0, xr::geom_from(geom), angles, nview, offsets, counts, rows, cols, vals, workspace,
                      workspace_bytes, stream);
}

int xr_sysmat3d(const xr_geom3d* geom, const float* angles, int nview, const long long* offsets, long long* counts,
                long long* rows, long long* cols, float* vals, void* workspace, size_t workspace_bytes, void* stream) {
    xr::Trace tr("xr_sysmat3d");
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    return xr::sysmat(1, xr::geom_from(geom), angles, nview, offsets, counts, rows, cols, vals, workspace,
                      workspace_bytes, stream);
}

int xr_ragged2d_plan_create(const xr_ragged2d_instance* inst, int ninst, xr_ragged2d_plan** plan,
                            size_t* workspace_bytes) {
    using namespace xr;
    if (!inst || !plan || !workspace_bytes || ninst < 1) return fail(XR_ERR_INVALID_ARGUMENT, "bad ragged plan arguments");
    auto* P = new xr_ragged2d_plan();
    P->inst.assign(inst, inst + ninst);
    P->max_nu = 0;
    size_t o = 0;
    RaggedLayout& L = P->lay;
    L.desc = o; o = align256(o + (size_t)ninst * sizeof(RaggedDev));
    L.sync = o; o = align256(o + 64);
    long long tot[10] = {0};
    for (int i = 0; i < ninst; ++i) {
        const Geom g = geom_from(&inst[i].geom);
        const int V = inst[i].nview;
        if (int rc = validate(g, 0, OP_A, 1, V)) { delete P; return rc; }
        if (V < 1) { delete P; return fail(XR_ERR_INVALID_ARGUMENT, "instance %d has no views", i); }
        if ((long long)g.H * g.W > (1ll << 30)) { delete P; return fail(XR_ERR_UNSUPPORTED, "instance %d image too large", i); }
        P->geom.push_back(g);
        P->max_nu = std::max(P->max_nu, g.Nu);
        std::array<int, 10> st{};
        for (int l = 0; l < 10; ++l) {
            st[l] = (int)tot[l];
            tot[l] += ragged_tiles(g, V, l);
        }
        P->starts.push_back(st);
        const size_t Vs = (size_t)V;
        L.hdr.push_back(o);  o = align256(o + Vs * sizeof(ViewHdr));
        L.bA.push_back(o);   o = align256(o + Vs * (g.Nu + 1) * sizeof(double));
        L.bB.push_back(o);   o = align256(o + Vs * (g.Nu + 1) * sizeof(double));
        L.colQ.push_back(o); o = align256(o + Vs * g.Nu * sizeof(double));
        L.colR.push_back(o); o = align256(o + Vs * g.Nu * sizeof(double));
        L.colE.push_back(o); o = align256(o + Vs * g.Nu * sizeof(float));
        L.colF.push_back(o); o = align256(o + Vs * g.Nu * sizeof(float));
        L.colM.push_back(o); o = align256(o + Vs * g.Nu * sizeof(float));
        L.arc.push_back(o);
        if (g.type == GEO_ARC) o = align256(o + 2 * Vs * (g.Nu + 1) * sizeof(float4));  // Bw's chained walks
        L.imgT.push_back(o); o = align256(o + (size_t)g.H * g.W * sizeof(float));
        L.filt.push_back(o); o = align256(o + Vs * g.Nu * sizeof(float));
    }
    for (int l = 0; l < 10; ++l) {
        if (tot[l] > 0x7fffffffll) { delete P; return fail(XR_ERR_UNSUPPORTED, "ragged batch too large"); }
        P->totals[l] = (int)tot[l];
    }
    L.total = o;
    P->smem = std::max<size_t>(256, 3 * (size_t)P->max_nu + 16) * sizeof(float);
    if (P->smem > 200 * 1024) { delete P; return fail(XR_ERR_UNSUPPORTED, "detector too wide for the ragged kernel"); }
    if (cudaGetDevice(&P->device) != cudaSuccess) { delete P; return fail(XR_ERR_CUDA, "cudaGetDevice failed"); }
    if (P->smem > 48 * 1024 &&
        cudaFuncSetAttribute(ragged2d_fbp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P->smem) != cudaSuccess) {
        delete P; return fail(XR_ERR_CUDA, "cannot reserve shared memory");
    }
    int per_sm = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ragged2d_fbp_kernel, 256, P->smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P->device) != cudaSuccess || per_sm < 1) {
        delete P; return fail(XR_ERR_CUDA, "occupancy query failed");
    }
    P->grid = per_sm * nsm;
    P->workspace = nullptr;
    *plan = P;
    *workspace_bytes = L.total;
    return XR_OK;
}

int xr_ragged2d_plan_bind(xr_ragged2d_plan* P, const float* images, float* sino, float* recon, const float* angles,
                          const float* filt, const float* cosw, void* workspace, size_t workspace_bytes) {
    using namespace xr;
    if (!P || !images || !sino || !recon || !angles || !filt || !cosw || !workspace)
        return fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    if (workspace_bytes < P->lay.total) return fail(XR_ERR_WORKSPACE, "workspace of %zu bytes required", P->lay.total);
    if (reinterpret_cast<uintptr_t>(workspace) % 256) return fail(XR_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    char* ws = static_cast<char*>(workspace);
    const RaggedLayout& L = P->lay;
    std::vector<RaggedDev> d(P->inst.size());
    for (size_t i = 0; i < d.size(); ++i) {
        const xr_ragged2d_instance& in = P->inst[i];
        RaggedDev& r = d[i];
        r.g = P->geom[i];
        r.vt.hdr = reinterpret_cast<ViewHdr*>(ws + L.hdr[i]);
        r.vt.bA = reinterpret_cast<double*>(ws + L.bA[i]);
        r.vt.bB = reinterpret_cast<double*>(ws + L.bB[i]);
        r.vt.colQ = reinterpret_cast<double*>(ws + L.colQ[i]);
        r.vt.colR = reinterpret_cast<double*>(ws + L.colR[i]);
        r.vt.colE = reinterpret_cast<float*>(ws + L.colE[i]);
        r.vt.colF = reinterpret_cast<float*>(ws + L.colF[i]);
        r.vt.colM = reinterpret_cast<float*>(ws + L.colM[i]);
        r.vt.hel = nullptr;
        r.vt.arc = r.g.type == GEO_ARC ? reinterpret_cast<float4*>(ws + L.arc[i]) : nullptr;
        r.vt.colWR = nullptr;
        r.nview = in.nview;
        r.cw = column_width(r.g, 0);
        r.scale = in.scale;
        r.img = images + in.img_offset;
        r.imgT = reinterpret_cast<float*>(ws + L.imgT[i]);
        r.sino = sino + in.sino_offset;
        r.filt_out = reinterpret_cast<float*>(ws + L.filt[i]);
        r.recon = recon + in.img_offset;
        r.ang = angles + in.ang_offset;
        r.filt = filt + in.filt_offset;
        r.cosw = cosw + in.cosw_offset;
        for (int l = 0; l < 10; ++l) r.t0[l] = P->starts[i][l];
    }
    if (cudaMemcpy(ws + L.desc, d.data(), d.size() * sizeof(RaggedDev), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(ws + L.sync, 0, 64) != cudaSuccess)
        return fail(XR_ERR_CUDA, "descriptor upload failed");
    P->workspace = workspace;
    return XR_OK;
}

int xr_ragged2d_run(const xr_ragged2d_plan* P, int project, int a_cols_log2, int view_split_log2, void* stream) {
    using namespace xr;
    Trace tr("xr_ragged2d_run");
    if (!P || !P->workspace) return fail(XR_ERR_INVALID_ARGUMENT, "plan not bound to a workspace");
    if (a_cols_log2 < 0 || a_cols_log2 > 3 || view_split_log2 < 0 || view_split_log2 > 3)
        return fail(XR_ERR_INVALID_ARGUMENT, "tile parameters out of range");
    char* ws = static_cast<char*>(P->workspace);
    const RaggedDev* desc = reinterpret_cast<const RaggedDev*>(ws + P->lay.desc);
    unsigned* bar = reinterpret_cast<unsigned*>(ws + P->lay.sync);
    int* ctr = reinterpret_cast<int*>(ws + P->lay.sync + 16);
    const int4 totals = make_int4(P->totals[0], project ? P->totals[2 + a_cols_log2] : 0, P->totals[1],
                                  P->totals[6 + view_split_log2]);
    const int4 lists = make_int4(0, 2 + a_cols_log2, 1, 6 + view_split_log2);
    const int ninst = (int)P->inst.size();
    const int CW = 32 << a_cols_log2, VS = 1 << view_split_log2;
    // barrier word and tile counters start at zero on every launch (also in
    // a captured graph), even after a launch whose barrier gave up
    if (cudaMemsetAsync(ws + P->lay.sync, 0, 64, static_cast<cudaStream_t>(stream)) != cudaSuccess)
        return fail(XR_ERR_CUDA, "resetting the ragged kernel's sync words failed");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P->grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = P->smem;
    cfg.stream = static_cast<cudaStream_t>(stream);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, ragged2d_fbp_kernel, desc, ninst, totals, lists, project, CW, VS, bar, ctr) !=
        cudaSuccess)
        return check_cuda("ragged2d_fbp (cooperative launch)");
    return check_cuda("ragged2d_fbp");
}

int xr_ragged2d_plan_info(const xr_ragged2d_plan* P, int* grid, int* tiles10) {
    if (!P || !grid || !tiles10) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    *grid = P->grid;
    for (int l = 0; l < 10; ++l) tiles10[l] = P->totals[l];
    return XR_OK;
}

void xr_ragged2d_plan_destroy(xr_ragged2d_plan* plan) { delete plan; }

int xr_ctpd_load(const char* const* paths, int nfiles, int rows, int cols, int col_stride, int row_stride,
                 int nthreads, float* sino, float* views, int* failed_file) {
    xr::Trace tr("xr_ctpd_load");
    if (failed_file) *failed_file = -1;
    if (!paths || !sino || !views || nfiles < 1 || rows < 1 || cols < 1 || col_stride < 1 || row_stride < 1)
        return xr::fail(XR_ERR_INVALID_ARGUMENT, "xr_ctpd_load: null pointer or non-positive size");
    for (int i = 0; i < nfiles; ++i)
        if (!paths[i]) return xr::fail(XR_ERR_INVALID_ARGUMENT, "xr_ctpd_load: null path %d", i);
    ctpd::Job job;
    job.paths = paths;
    job.nfiles = nfiles;
    job.rows = rows;
    job.cols = cols;
    job.cs = col_stride;
    job.rs = row_stride;
    job.nv = (cols + row_stride - 1) / row_stride;
    job.nu = (rows + col_stride - 1) / col_stride;
    job.sino = sino;
    job.views = views;
    int T = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
    T = std::max(1, std::min({T, nfiles, 64}));
    std::vector<std::thread> pool;
    pool.reserve(T - 1);
    try {
        for (int t = 1; t < T; ++t) pool.emplace_back(ctpd::worker, &job);
    } catch (const std::exception&) {
        // fewer threads than asked: the ones started and this one share the files
    }
    ctpd::worker(&job);
    for (auto& th : pool) th.join();
    const int bad = job.failed.load();
    if (bad >= 0) {
        if (failed_file) *failed_file = bad;
        return xr::fail(XR_ERR_UNSUPPORTED, "xr_ctpd_load: file %d (%s) is not a file this reader takes", bad,
                        paths[bad]);
    }
    return XR_OK;
}

const char* xr_version(void) { return "xrecon_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
