// C ABI of libxrecon_b200.so: validation, workspace layout and launches.
// The declarations and the reference interface each call replaces are in
// include/xrecon_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "xr_kernels.cuh"
#include "../../include/xrecon_b200.h"

namespace xr {
namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int check_cuda(const char* what) {
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
    size_t hdr, bA, bB, colQ, colE, colF, colM, volT, sinoS, total;
};

// Image-input ops of the cell gather need the flipped transpose of the image
// (lines of y-axis views); cone A^T needs an FP32 pre-scaled sinogram.
Layout layout(int dim3d, int op, const Geom& g, int nbatch, int nview, int dtype_in) {
    Layout l{};
    size_t o = 0;
    const size_t V = (size_t)(nview > 0 ? nview : 1);
    l.hdr = o;   o = align256(o + V * sizeof(ViewHdr));
    l.bA = o;    o = align256(o + V * (g.Nu + 1) * sizeof(double));
    l.bB = o;    o = align256(o + V * (g.Nu + 1) * sizeof(double));
    l.colQ = o;  o = align256(o + V * g.Nu * sizeof(double));
    l.colE = o;  o = align256(o + V * g.Nu * sizeof(float));
    l.colF = o;  o = align256(o + V * g.Nu * sizeof(float));
    l.colM = o;  o = align256(o + V * g.Nu * sizeof(float));
    int eff = op;
    if (g.type == GEO_PARALLEL && dim3d) {
        if (op == OP_B || op == OP_BW) eff = OP_AT;
        else if (op == OP_BT || op == OP_BWT) eff = OP_A;
    }
    l.volT = o;
    if (eff == OP_A || eff == OP_BT || eff == OP_BWT)
        o = align256(o + (size_t)nbatch * g.D * g.H * g.W * dtype_size(dtype_in));
    l.sinoS = o;
    if (dim3d && eff == OP_AT && g.type != GEO_PARALLEL)
        o = align256(o + (size_t)nbatch * V * g.Nv * g.Nu * sizeof(float));
    l.total = o;
    return l;
}

ViewTables tables_at(char* ws, const Layout& l) {
    ViewTables t;
    t.hdr = reinterpret_cast<ViewHdr*>(ws + l.hdr);
    t.bA = reinterpret_cast<double*>(ws + l.bA);
    t.bB = reinterpret_cast<double*>(ws + l.bB);
    t.colQ = reinterpret_cast<double*>(ws + l.colQ);
    t.colE = reinterpret_cast<float*>(ws + l.colE);
    t.colF = reinterpret_cast<float*>(ws + l.colF);
    t.colM = reinterpret_cast<float*>(ws + l.colM);
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

constexpr int CELL_R = 8;
constexpr int VOX_R = 16;
constexpr int VOX_NW = 4;

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
        TI* volT = reinterpret_cast<TI*>(ws + l.volT);
        dim3 tg((g.W + 31) / 32, (g.H + 31) / 32, g.D * nbatch);
        transpose_flip_kernel<TI><<<tg, dim3(32, 8), 0, st>>>(in, volT, g.H, g.W);
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
    const float uscale = (g.type == GEO_FLAT) ? (float)(g.sod / g.sdd) : 1.0f;
    const float atconst = (float)(g.dx * g.dy * g.dz / (g.du * g.dv));
    if (eff == OP_AT) {
        if (g.type != GEO_PARALLEL) {
            float* sinoS = reinterpret_cast<float*>(ws + l.sinoS);
            const size_t total = (size_t)nbatch * nview * g.Nv * g.Nu;
            prescale_at3d_kernel<TI><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(g, vt, in, sinoS, nview, total, zd0, dvv);
            if (int rc = check_cuda("prescale_at3d")) return rc;
            vox_gather3d_kernel<float, TO, VOX_R, OP_AT><<<grid, block, 0, st>>>(
                g, vt, sinoS, out, nview, nzg, z0dz, zd0, dvv, cw, uscale, atconst, oscale);
        } else {
            vox_gather3d_kernel<TI, TO, VOX_R, OP_AT><<<grid, block, 0, st>>>(
                g, vt, in, out, nview, nzg, z0dz, zd0, dvv, cw, uscale, atconst, oscale);
        }
    } else if (eff == OP_B) {
        vox_gather3d_kernel<TI, TO, VOX_R, OP_B><<<grid, block, 0, st>>>(
            g, vt, in, out, nview, nzg, z0dz, zd0, dvv, cw, uscale, atconst, oscale);
    } else {
        vox_gather3d_kernel<TI, TO, VOX_R, OP_BW><<<grid, block, 0, st>>>(
            g, vt, in, out, nview, nzg, z0dz, zd0, dvv, cw, uscale, atconst, oscale);
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
        transpose_flip_kernel<TI><<<tg, dim3(32, 8), 0, st>>>(in, imgT, g.H, g.W);
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
    if (!in || !out) return fail(XR_ERR_INVALID_ARGUMENT, "null input or output pointer");
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

}  // namespace
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
    return xr::layout(1, op, g, nbatch, nview, xr::DT_F32).total;
}

int xr_dd2d(int op, const xr_geom2d* geom, const void* in, int dtype_in, void* out, int dtype_out,
            const float* angles, int nbatch, int nview, void* workspace, size_t workspace_bytes,
            void* stream) {
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    return xr::apply(0, op, xr::geom_from(geom), in, dtype_in, out, dtype_out, angles, nbatch, nview,
                     workspace, workspace_bytes, stream, 1.0f);
}

int xr_dd3d(int op, const xr_geom3d* geom, const void* in, int dtype_in, void* out, int dtype_out,
            const float* angles, int nbatch, int nview, void* workspace, size_t workspace_bytes,
            void* stream) {
    if (!geom) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null geometry");
    return xr::apply(1, op, xr::geom_from(geom), in, dtype_in, out, dtype_out, angles, nbatch, nview,
                     workspace, workspace_bytes, stream, 1.0f);
}

int xr_fbp_filter(const void* in, int dtype_in, float* out, int nrows, int Nu, int nview, int rows_per_view,
                  const float* cosw, const float* filt, const float* parker, void* stream) {
    if (!in || !out || !filt) return xr::fail(XR_ERR_INVALID_ARGUMENT, "null pointer");
    if (Nu < 1 || nrows < 0 || nview < 1 || rows_per_view < 1)
        return xr::fail(XR_ERR_INVALID_ARGUMENT, "bad filter sizes");
    if (nrows == 0) return XR_OK;
    if (!xr::dtype_ok(dtype_in)) return xr::fail(XR_ERR_INVALID_ARGUMENT, "unsupported dtype %d", dtype_in);
    constexpr int OUTS = 8;
    const size_t smem = (size_t)(3 * Nu + 2 * OUTS) * sizeof(float);
    if (smem > 200 * 1024) return xr::fail(XR_ERR_UNSUPPORTED, "detector width %d too large for the filter kernel", Nu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = std::min(nrows, 148 * 8);
    if (dtype_in == xr::DT_F32) {
        auto k = xr::fbp_filter_kernel<float, OUTS>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, 256, smem, st>>>(static_cast<const float*>(in), out, nrows, Nu, nview, rows_per_view, cosw, filt, parker);
    } else if (dtype_in == xr::DT_BF16) {
        auto k = xr::fbp_filter_kernel<__nv_bfloat16, OUTS>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, 256, smem, st>>>(static_cast<const __nv_bfloat16*>(in), out, nrows, Nu, nview, rows_per_view, cosw, filt, parker);
    } else {
        auto k = xr::fbp_filter_kernel<__half, OUTS>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, 256, smem, st>>>(static_cast<const __half*>(in), out, nrows, Nu, nview, rows_per_view, cosw, filt, parker);
    }
    return xr::check_cuda("fbp_filter");
}

const char* xr_last_error(void) { return xr::g_last_error.c_str(); }

const char* xr_version(void) { return "xrecon_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
