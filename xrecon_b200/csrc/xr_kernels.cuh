// Kernels of the B200 distance-driven projector.
//
// Two gather shapes cover all six operators of each geometry (so no kernel
// needs atomics):
//   cell gather (detector-cell owned):  A, B^T, Bw^T
//       y[cell] = S_cell * sum_vox K[cell, vox] * T_vox * x[vox]
//   voxel gather (voxel owned):         A^T, B, Bw
//       x[vox]  = sum_views T_vox * sum_cells K[cell, vox] * S_cell * y[cell]
// with S_cell = s_A (A, A^T) or 1, and T_vox = column width (B family), times
// the FBP voxel weight for Bw.
//
// Reference kernels these replace (XRecon src/kernels): forward3d_flat.cu:7-246
// and forward3d_arc.cu:7-243 (A), backward3d_flat.cu:7-128 and
// backward3d_arc.cu:7-128 (B/Bw), forward3d_flat.cu:249-486 and
// forward3d_arc.cu:246-480 (A^T), backward3d_flat.cu:131-377 and
// backward3d_arc.cu:131-249 (B^T/Bw^T), forward3d_parallel.cu:33-219 (3D
// parallel), forward2d.cu / forward2d_t.cu / backward2d.cu / backward2d_t.cu
// (2D).
#pragma once

#include "xr_common.cuh"

namespace xr {

constexpr int MAXB = 4;  // pixels per column handled per merge pass

// Sum over the pixel band of one column: sum_i w[i] * vol[j, L, pc + i].
template <typename TI>
__device__ __forceinline__ float band_value(const TI* __restrict__ base, int j, size_t plane, int D,
                                            const float (&w)[MAXB], int np) {
    if ((unsigned)j >= (unsigned)D) return 0.0f;
    const TI* p = base + (size_t)j * plane;
    float s = w[0] * ld(p);
#pragma unroll
    for (int i = 1; i < MAXB; ++i)
        if (i < np) s = fmaf(w[i], ld(p + i), s);
    return s;
}

// Same sum at a pointer already positioned on voxel row j of the band.
template <typename TI, int NB>
__device__ __forceinline__ float band_at(const TI* __restrict__ p, const float (&w)[NB], int np) {
    float s = w[0] * ld(p);
#pragma unroll
    for (int i = 1; i < NB; ++i)
        if (i < np) s = fmaf(w[i], ld(p + i), s);
    return s;
}

template <typename TI>
__device__ __forceinline__ float row_value(const TI* __restrict__ colbase, int m, int Nv, int Nu) {
    if ((unsigned)m >= (unsigned)Nv) return 0.0f;
    return ld(colbase + (size_t)m * Nu);
}

// ------------------------------------------------------------------ setup

// One thread per (view, boundary k in 0..Nu).  FP64 throughout, except the
// float32 boundary angles of circular arc detectors (arcf; see arc_angle_f).
__device__ __forceinline__ void setup_view_entry(const Geom& g, const int dim3d, const float angle, const int v,
                                                 const int k, const ViewTables& vt, const bool arcf = false);

__global__ void setup_views_kernel(const Geom g, const int dim3d, const float* __restrict__ ang,
                                   const int nview, const ViewTables vt) {
    const int v = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nview || k > g.Nu) return;
    setup_view_entry(g, dim3d, ang[v], v, k, vt, g.type == GEO_ARC);
}

// Axis position of arc boundary k with the reference's float32 rounding, and
// its two entries of ViewTables::arc (see there).
__device__ __forceinline__ double arc_boundary_f(const Geom& g, const ViewHdr& h, int k, float angle, float4& ea,
                                                 float4& eb) {
    const float tk = arc_angle_f(g, h.keep, (float)k, angle);
    const double T = tan((double)tk);
    const float hi = __double2float_rn(T);
    const float lo = __double2float_rn(T - (double)hi);
    const float Df = arc_axis_f(h, hi);
    // derivative of the axis map: x axis sy (1 + T^2), y axis -sx (1 + T^2) / T^2
    const double sec2 = 1.0 + T * T;
    const double dD = h.use_x ? (double)h.syf * sec2 : -(double)h.sxf * sec2 / (T * T);
    ea = make_float4(tk, (float)dD, 0.0f, 0.0f);  // .z, .w: the column width, filled by the caller
    eb = make_float4(Df, hi, lo, 0.0f);
    return (double)Df;
}

// Per-view tables of view v, boundary / column k (k = 0..Nu).
__device__ __forceinline__ void setup_view_entry(const Geom& g, const int dim3d, const float angle, const int v,
                                                 const int k, const ViewTables& vt, const bool arcf) {
    ViewHdr h;
    make_view_hdr(g, angle, h);
    if (k == 0) vt.hdr[v] = h;

    const double uscale = (dim3d && g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
    const size_t ob = (size_t)v * (g.Nu + 1) + k;
    float4 ea, eb;
    const double Dk = arcf ? arc_boundary_f(g, h, k, angle, ea, eb) : boundary_axis(g, h, (double)k, uscale);
    double A, B;
    boundary_line_coeffs(g, h, Dk, A, B);
    if (arcf && vt.arc) {
        if (k > 0) {
            // boundary k - 1 as its own thread evaluates it
            float4 pa, pb;
            double Ap, Bp;
            boundary_line_coeffs(g, h, arc_boundary_f(g, h, k - 1, angle, pa, pb), Ap, Bp);
            ea.z = (float)(A - Ap);
            ea.w = (float)(B - Bp);
        }
        vt.arc[2 * ob] = ea;
        vt.arc[2 * ob + 1] = eb;
    }
    vt.bA[ob] = A;
    vt.bB[ob] = B;
    if (k >= g.Nu) return;

    const size_t oc = (size_t)v * g.Nu + k;
    const double Dk1 = arcf ? arc_boundary_f(g, h, k + 1, angle, ea, eb) : boundary_axis(g, h, (double)k + 1.0, uscale);
    auto put_R = [&](double R) {
        vt.colR[oc] = R;
        if (vt.colWR) {
            double A1, B1;
            boundary_line_coeffs(g, h, Dk1, A1, B1);
            const float hi = (float)R;
            vt.colWR[oc] = make_float4((float)(A1 - A), (float)(B1 - B), hi, (float)(R - (double)hi));
        }
    };
    const double dperp = h.use_x ? g.dy : g.dx;
    if (g.type == GEO_PARALLEL) {
        // forward3d.cpp:58,98 (xy_scale / dv) and system_matrix2d.cpp:109.
        vt.colQ[oc] = 1.0 / g.dz;
        put_R(g.dz);
        vt.colE[oc] = (float)(dim3d ? dperp / (g.du * g.dv) : dperp / g.du);
        vt.colF[oc] = 1.0f;
        vt.colM[oc] = 0.0f;
        return;
    }
    double M;
    if (arcf) {
        // column centre at the float32 centre angle (forward3d.cpp:285-297)
        const double ac = (double)arc_angle_f(g, h.keep, (float)k + 0.5f, angle);
        const double cx = sin(ac) * g.sdd + h.sx, cy = -cos(ac) * g.sdd + h.sy;
        M = h.use_x ? h.sy / (h.sy - cy) : h.sx / (h.sx - cx);
    } else {
        M = column_mag(g, h, k, uscale);
    }
    vt.colQ[oc] = M / g.dz;
    put_R(g.dz / M);
    const double aa = 0.5 * (Dk + Dk1) - h.spar;
    const double F = aa * aa + h.sperp * h.sperp;
    if (dim3d) {
        // s_A = dperp / (area * triangle_cosine): forward3d.cpp:331-343.
        const double rs = (g.type == GEO_FLAT) ? g.sod / g.sdd : 1.0;
        vt.colE[oc] = (float)(dperp / (fabs(h.sperp) * (Dk1 - Dk) * M * g.dv * rs));
        vt.colF[oc] = (float)F;
        vt.colM[oc] = (float)M;
    } else {
        // 2D: dperp / ((D1 - D0) * cos_weight), system_matrix2d.cpp:213,251.
        vt.colE[oc] = (float)(dperp * sqrt(F) / (fabs(h.sperp) * (Dk1 - Dk)));
        vt.colF[oc] = 1.0f;
        vt.colM[oc] = 0.0f;
    }
}

// Image plane transpose with the y flip: out[b][x][H-1-y] = in[b][y][x], so
// that lines of the y-axis views (image columns) are contiguous in the
// pixel coordinate p = H-1-iy.
template <typename T>
__global__ void transpose_flip_kernel(const T* __restrict__ in, T* __restrict__ out, int H, int W, int pitch) {
    __shared__ T tile[32][33];
    const size_t plane = (size_t)H * W;
    const T* src = in + (size_t)blockIdx.z * plane;
    T* dst = out + (size_t)blockIdx.z * ((size_t)W * pitch);
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int y = y0 + dy, x = x0 + threadIdx.x;
        if (y < H && x < W) tile[dy][threadIdx.x] = src[(size_t)y * W + x];
    }
    __syncthreads();
    for (int dx = threadIdx.y; dx < 32; dx += blockDim.y) {
        const int x = x0 + dx, y = y0 + threadIdx.x;
        if (y < H && x < W) dst[(size_t)x * pitch + (H - 1 - y)] = tile[threadIdx.x][dx];
    }
}

// Half-precision image to FP32.  With both pointers 16-byte aligned a
// thread converts 8 elements (one 16-byte load, two 16-byte stores), so each
// thread keeps a whole sector in flight; otherwise element for element.
template <typename T>
__global__ void widen_kernel(const T* __restrict__ in, float* __restrict__ out, const size_t n, const bool vec) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (!vec) {
        if (i < n) out[i] = ld(in + i);
        return;
    }
    const size_t e = i * 8;
    if (e + 8 <= n) {
        static_assert(sizeof(T) == 2, "8 half-precision elements per 16-byte load");
        union { uint4 u; T h[8]; } p;
        p.u = __ldg(reinterpret_cast<const uint4*>(in + e));
        float f[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) f[j] = to_f(p.h[j]);
        float4* o = reinterpret_cast<float4*>(out + e);
        o[0] = make_float4(f[0], f[1], f[2], f[3]);
        o[1] = make_float4(f[4], f[5], f[6], f[7]);
    } else {
        for (size_t j = e; j < n; ++j) out[j] = ld(in + j);
    }
}

// Copy image planes into a row pitch that is a multiple of 16 bytes (TMA
// stride rule); the padding columns are never read inside the image.
template <typename T>
__global__ void pad_rows_kernel(const T* __restrict__ in, T* __restrict__ out, int W, int pitch, size_t nrows) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t row = i / W;
    if (row >= nrows) return;
    const int x = (int)(i % W);
    out[row * pitch + x] = in[i];
}

// Arc detector, cell-owned B^T / Bw^T: bounds of column k over the band's
// first pixel pa of line L when that pixel starts left of the column
// (pk > pa).  The reference walks that pixel's columns from the one holding
// its first edge, k0 < k, with chained angles (ArcChain): column k spans the
// chain's boundaries k and k + 1, s - 1 and s steps from k0.  u0, u1 are
// written relative to pa; qd converts axis offsets to pixels on line L.
__device__ __forceinline__ void arc_first_pixel_bounds(const Geom& g, const ViewTables& vt, const ViewHdr& h,
                                                       const float4* __restrict__ ea, int v, int k, int L, int pa,
                                                       double pk, double pk1, float qd, float& u0, float& u1) {
    const int Nu = g.Nu;
    const double* __restrict__ bA = vt.bA + (size_t)v * (Nu + 1);
    const double* __restrict__ bB = vt.bB + (size_t)v * (Nu + 1);
    int k0 = k - 1;
    while (k0 > 0 && fma(bB[k0], (double)L, bA[k0]) > (double)pa) --k0;
    ArcChain ch;
    ch.start(ea, k0, h.keep, (float)g.du);
    for (int j = k0 + 1; j < k; ++j) ch.t = __fadd_rn(ch.t, ch.step);
    const float dk = ch.next_exact(h, ea, k);
    float dk1 = ch.next_exact(h, ea, k + 1);
    if (k + 1 == Nu) dk1 = fminf(dk1, 0.0f);
    u0 = fmaf(dk, qd, (float)(pk - (double)pa));
    u1 = fmaf(dk1, qd, (float)(pk1 - (double)pa));
}

// ------------------------------------------------------------- 3D kernels

// Cell gather: lane = detector column (traversal order), warp = run of R
// detector rows.  Each thread sweeps the image lines; per line it forms the
// pixel band of its column (FP64 boundaries, FP32 weights) and merges the
// z voxels of the band against its R rows in local coordinates.
template <typename TI, typename TO, int R, int MODE, bool HEL = false>
__global__ void __launch_bounds__(256, 3)
cell_gather3d_kernel(const Geom g, const ViewTables vt, const TI* __restrict__ vol_rows,
                     const TI* __restrict__ vol_cols, TO* __restrict__ sino, const int nview,
                     const int view0, const double z0dz_p, const double zd0_p, const double dvv,
                     const float cw_p) {
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int r0 = (blockIdx.y * blockDim.y + threadIdx.y) * R;
    const int vb = blockIdx.z + view0;
    const int v = vb % nview, b = vb / nview;
    const int Nu = g.Nu;
    if (k >= Nu || r0 >= g.Nv) return;
    const ViewHdr h = vt.hdr[v];
    // helical scans: the view's own z placement and column width
    const double z0dz = HEL ? vt.hel[v].z0dz : z0dz_p;
    const double zd0 = HEL ? vt.hel[v].zd0 : zd0_p;
    const float cw = HEL ? vt.hel[v].cw : cw_p;
    const size_t ob = (size_t)v * (Nu + 1) + k;
    const double bA0 = vt.bA[ob], bB0 = vt.bB[ob], bA1 = vt.bA[ob + 1], bB1 = vt.bB[ob + 1];
    const double Qk = vt.colQ[(size_t)v * Nu + k];
    const int nlines = h.nlines, npix = h.npix;
    const size_t plane = (size_t)nlines * npix;
    const TI* __restrict__ vol = (h.use_x ? vol_rows : vol_cols) + (size_t)b * g.D * plane;
    const double zr0 = zd0 + r0 * dvv;
    // arc detector, B^T / Bw^T: chained column walks (see cell2d_sum)
    const bool chain = (MODE == OP_BT || MODE == OP_BWT) && !HEL && vt.arc;
    const float4* __restrict__ ea = chain ? vt.arc + 2 * (size_t)v * (Nu + 1) : nullptr;
    float d1 = 0.0f;
    if (chain) {
        ArcChain ch;
        ch.start(ea, k, h.keep, (float)g.du);
        d1 = ch.next_exact(h, ea, k + 1);
        if (k + 1 == Nu) d1 = fminf(d1, 0.0f);
    }

    float acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = 0.0f;

    const float dpdz = (float)(h.dpix * g.dz);
    for (int L = 0; L < nlines; ++L) {
        const double pk = fma(bB0, (double)L, bA0);
        const double pk1 = fma(bB1, (double)L, bA1);
        const int pa = max((int)floor(pk), 0);
        const int pb = min((int)ceil(pk1) - 1, npix - 1);
        if (pa > pb) continue;
        const double q = fma(h.q1, (double)L, h.q0);
        const double gq = Qk * q;
        const double t0 = fma(gq, zr0, -z0dz);
        const double bt = gq * dvv;
        if (!(bt > 1.0e-4 && bt < 1.0e4)) continue;  // bounds every merge loop
        if (t0 + R * bt <= 0.0 || t0 >= (double)g.D) continue;
        const double jf = floor(t0);
        const int j0 = (int)jf;
        const float f = (float)(t0 - jf);
        const float bf = (float)bt;
        float lf = cw;
        if (MODE == OP_A) {
            const float qf = (float)q;
            lf = dpdz / (qf * qf);
        }
        // band edges relative to the first pixel: small FP32 numbers
        float u0 = (float)(pk - (double)pa), u1 = (float)(pk1 - (double)pa);
        float u1b = u1;  // upper edge for the band's later pixels
        if (chain) {
            const float qd = (float)(q / h.dpix);
            u1b = fmaf(d1, qd, u1);
            u1 = u1b;
            if (k > 0 && pk > (double)pa)
                arc_first_pixel_bounds(g, vt, h, ea, v, k, L, pa, pk, pk1, qd, u0, u1);
        }
        const TI* __restrict__ line = vol + (size_t)L * npix;
        for (int pc = pa; pc <= pb; pc += MAXB) {
            const int np = min(MAXB, pb - pc + 1);
            const float off = (float)(pc - pa);
            float w[MAXB];
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                float wi = 0.0f;
                if (i < np) {
                    wi = (fminf(off + (float)(i + 1), (pc + i == pa) ? u1 : u1b) - fmaxf(off + (float)i, u0)) * lf;
                    if (MODE == OP_BWT) {
                        float px, py;
                        pixel_center(g, h, L, pc + i, px, py);
                        wi *= fbp_weight(g, h, px, py);
                    }
                }
                w[i] = wi;
            }
            // Voxel walk in local z coordinates (voxel j0+m spans [m, m+1]).
            // Below the volume a single virtual zero voxel ends at voxel 0;
            // past the top the value is zero and the next boundary infinite.
            const TI* __restrict__ ptr;
            int jabs;
            float vj, jn;
            float pos = f;
            if (j0 >= 0) {
                jabs = j0;
                ptr = line + (size_t)j0 * plane + pc;
                vj = band_at(ptr, w, np);
                jn = 1.0f;
            } else {
                // address of "voxel -1": only ever advanced to voxel 0, never read
                jabs = -1;
                ptr = line + pc - plane;
                vj = 0.0f;
                jn = (float)(-j0);
            }
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const float top = fmaf(bf, (float)(i + 1), f);
                float a = 0.0f;
                while (jn < top) {
                    a = fmaf(jn - pos, vj, a);
                    pos = jn;
                    ++jabs;
                    ptr += plane;
                    if (jabs < g.D) { vj = band_at(ptr, w, np); jn += 1.0f; }
                    else { vj = 0.0f; jn = 3.0e38f; }
                }
                if (top > pos) { a = fmaf(top - pos, vj, a); pos = top; }
                acc[i] += a;
            }
        }
    }

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
            float s = acc[i];
            if (MODE == OP_A) {
                float zc = (float)(zd0 + (r + 0.5) * dvv) * M;
                if (HEL) zc += vt.hel[v].zsrc;  // helical: the row's absolute z
                s *= E * sqrtf(F + zc * zc);
            }
            st(out + (size_t)r * Nu, s);
        }
    }
}

// A^T cell scale applied to the sinogram once (cone geometries).
template <typename TI>
__global__ void prescale_at3d_kernel(const Geom g, const ViewTables vt, const TI* __restrict__ in,
                                     float* __restrict__ out, const int nview, const size_t total,
                                     const double zd0, const double dvv) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % g.Nu);
    const int r = (int)((idx / g.Nu) % g.Nv);
    const int v = (int)((idx / ((size_t)g.Nu * g.Nv)) % nview);
    const int keep = vt.hdr[v].keep;
    const int k = keep ? c : g.Nu - 1 - c;
    const size_t oc = (size_t)v * g.Nu + k;
    const float zc = (float)(zd0 + (r + 0.5) * dvv) * vt.colM[oc];
    out[idx] = ld(in + idx) * vt.colE[oc] * sqrtf(vt.colF[oc] + zc * zc);
}

// Float constants of the image grid and detector used by the FP32 column
// guess and the FBP weight (exactness comes from the FP64 tables).
struct GeomF {
    float x0, y0;      // left / bottom image edge
    float xc0, yc0;    // centre of column 0 / row 0 (row 0 is the top)
    float dx, dy;
    float sod, uscale, shu, du;
    float inv_uscale, inv_du;  // reciprocals for the column guess
    int H, Nu, type;
};

__device__ __forceinline__ float col_guess_f(const GeomF& gf, const ViewHdr& h, float x, float y) {
    const float s = (float)h.s, c = (float)h.c;
    float sg;
    if (gf.type == GEO_FLAT) {
        const float R = gf.sod;
        const float u = R * (x * c + y * s) / (R + x * s - y * c);
        sg = (u / gf.uscale - gf.shu) / gf.du;
    } else if (gf.type == GEO_ARC) {
        const float ac = (float)h.beta + gf.shu;
        float dcx, dcy;
        sincosf(ac, &dcx, &dcy);
        dcy = -dcy;
        const float ex = x - (float)h.sx, ey = y - (float)h.sy;
        sg = atan2f(dcx * ey - dcy * ex, dcx * ex + dcy * ey) / gf.du;
    } else {
        sg = (x * c + y * s - gf.shu) / gf.du;
    }
    return h.keep ? sg + 0.5f * gf.Nu : 0.5f * gf.Nu - sg;
}

// Voxel gather: lane = image column ix (32 consecutive), warp = run of R
// voxels along z.  Each thread sweeps all views; per view it finds the
// detector columns overlapping its pixel (FP32 guess widened by one column
// each side, exact FP64 boundaries) and merges its R voxels against the rows
// of each column: voxels are the static loop, rows the dynamic one.  Below
// the detector a single virtual zero row ends at row 0; past the top the
// value is zero and the next boundary infinite.
template <typename TI, typename TO, int R, int MODE>
__global__ void __launch_bounds__(128)
vox_gather3d_kernel(const Geom g, const GeomF gf, const ViewTables vt, const TI* __restrict__ sino,
                    TO* __restrict__ vol, const int nview, const int nzg, const double z0dz, const double zd0,
                    const double dvv, const float cw, const float atconst, const float oscale) {
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y;
    const int zg = blockIdx.z % nzg, b = blockIdx.z / nzg;
    const int j0 = (zg * blockDim.y + threadIdx.y) * R;
    if (ix >= g.W || j0 >= g.D) return;
    const int Nu = g.Nu, Nv = g.Nv;
    const float dpdz = (float)(g.dz);
    float acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = 0.0f;
    const TI* __restrict__ sinob = sino + (size_t)b * nview * Nv * Nu;
    const double dj0 = (double)j0;

    for (int v = 0; v < nview; ++v) {
        const ViewHdr& h = vt.hdr[v];
        const int use_x = h.use_x, keep = h.keep;
        int L, p;
        float xa, ya, xb, yb, px, py;
        if (use_x) {
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
        float lf;
        if (MODE == OP_AT) {
            if (g.type == GEO_PARALLEL) lf = atconst;
            else { const float qf = (float)q; lf = (float)h.dpix * dpdz / (qf * qf); }
        } else {
            lf = cw;
            if (MODE == OP_BW) lf *= fbp_weight(g, h, px, py);
        }
        lf *= oscale;
        const float kf0 = col_guess_f(gf, h, xa, ya), kf1 = col_guess_f(gf, h, xb, yb);
        const float lo = fmaxf(fminf(fminf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const float hi = fmaxf(fminf(fmaxf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const int ka = max(0, (int)floorf(lo) - 1);
        const int kb = min(Nu - 1, (int)floorf(hi) + 1);
        if (ka > kb) continue;
        const double* __restrict__ bA = vt.bA + (size_t)v * (Nu + 1);
        const double* __restrict__ bB = vt.bB + (size_t)v * (Nu + 1);
        const double* __restrict__ Q = vt.colQ + (size_t)v * Nu;
        const TI* __restrict__ sv = sinob + (size_t)v * Nv * Nu;
        const double dp = (double)p;
        // z merge of column k, overlapping the pixel by wf
        auto column = [&](const int k, const float wf) {
            const double gq = Q[k] * q;
            const double T0 = fma(gq, zd0, -z0dz);
            const double bt = gq * dvv;
            if (!(bt > 1.0e-4 && bt < 1.0e4)) return;  // bounds every merge loop
            if (T0 >= dj0 + R || T0 + Nv * bt <= dj0) return;
            const float bf = (float)bt;
            const int col = keep ? k : Nu - 1 - k;
            const TI* __restrict__ yp;
            int m;
            float y, rn;
            if (T0 > dj0) {
                // run starts below row 0: virtual zero row up to row 0
                m = -1;
                y = 0.0f;
                rn = (float)(T0 - dj0);
                yp = sv + col - Nu;  // address only; advanced to row 0 before any read
            } else {
                int rs = (int)floorf((float)(dj0 - T0) * __frcp_rn(bf));
                double trs = fma((double)rs, bt, T0);
                if (trs > dj0) { --rs; trs -= bt; }
                else if (trs + bt <= dj0) { ++rs; trs += bt; }
                if (rs > Nv - 1) { rs = Nv - 1; trs = fma((double)rs, bt, T0); }
                if (rs < 0) { rs = 0; trs = T0; }
                m = rs;
                yp = sv + col + (size_t)rs * Nu;
                y = ld(yp);
                rn = (float)(trs - dj0) + bf;
            }
            const float wk = wf * lf;
            float pos = 0.0f;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const float top = (float)(i + 1);
                float a = 0.0f;
                while (rn < top) {
                    a = fmaf(rn - pos, y, a);
                    pos = rn;
                    ++m;
                    yp += Nu;
                    if (m < Nv) { y = ld(yp); rn += bf; }
                    else { y = 0.0f; rn = 3.0e38f; }
                }
                a = fmaf(top - pos, y, a);
                pos = top;
                acc[i] = fmaf(wk, a, acc[i]);
            }
        };
        if (MODE != OP_AT && vt.arc) {
            // arc detector: the pixel's columns walked with chained angles
            const float4* __restrict__ ea = vt.arc + 2 * (size_t)v * (Nu + 1);
            const double qd = q / h.dpix;  // pixels per axis unit
            int k = ka;
            double pkl = fma(bB[k], (double)L, bA[k]);
            double pk1 = fma(bB[k + 1], (double)L, bA[k + 1]);
            while (!(pk1 > dp) && k < kb) {
                ++k;
                pkl = pk1;
                pk1 = fma(bB[k + 1], (double)L, bA[k + 1]);
            }
            ArcChain ch;
            ch.start(ea, k, h.keep, (float)g.du);
            for (;;) {
                float d = ch.next_linear(ea, k + 1);
                if (k + 1 == Nu) d = fminf(d, 0.0f);  // the detector's end
                pk1 = fma((double)d, qd, pk1);
                const float wf = (float)(fmin(dp + 1.0, pk1) - fmax(dp, pkl));
                if (wf > 0.0f) column(k, wf);
                if (++k > kb) break;
                pkl = pk1;
                if (pkl >= dp + 1.0) break;
                pk1 = fma(bB[k + 1], (double)L, bA[k + 1]);
            }
            continue;
        }
        double pk = fma(bB[ka], (double)L, bA[ka]);
        for (int k = ka; k <= kb; ++k) {
            const double pk1 = fma(bB[k + 1], (double)L, bA[k + 1]);
            const float wf = (float)(fmin(dp + 1.0, pk1) - fmax(dp, pk));
            pk = pk1;
            if (wf > 0.0f) column(k, wf);
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = j0 + i;
        if (j < g.D) st(vol + (((size_t)b * g.D + j) * g.H + iy) * g.W + ix, acc[i]);
    }
}

// ------------------------------------------------------------- 2D kernels

// Cell gather, 2D: one thread per (view, column).
template <typename TI, int MODE>
__device__ __forceinline__ float cell2d_sum(const Geom& g, const ViewTables& vt, const ViewHdr& h,
                                            const TI* __restrict__ img_rows, const TI* __restrict__ img_cols,
                                            const int v, const int k, const float cw, const int l0, const int ls);
template <typename TI, int MODE>
__device__ __forceinline__ float pix2d_sum(const Geom& g, const ViewTables& vt, const TI* __restrict__ sinob,
                                           const int ix, const int iy, const float cw, const int v0,
                                           const int v1, const int vs);

template <typename TI, typename TO, int MODE>
__global__ void __launch_bounds__(128)
cell_gather2d_kernel(const Geom g, const ViewTables vt, const TI* __restrict__ img_rows,
                     const TI* __restrict__ img_cols, TO* __restrict__ sino, const int nview,
                     const float cw) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y, b = blockIdx.z;
    const int Nu = g.Nu;
    if (k >= Nu) return;
    const ViewHdr h = vt.hdr[v];
    const size_t plane = (size_t)g.W * g.H;
    const float acc = cell2d_sum<TI, MODE>(g, vt, h, img_rows + b * plane, img_cols + b * plane, v, k, cw, 0, 1);
    const int col = h.keep ? k : Nu - 1 - k;
    st(sino + ((size_t)b * nview + v) * Nu + col, acc);
}

// Cell k of view v (traversal order), lines L = l0, l0 + ls, ...: the 2D DD
// line sum, times the cell scale colE for MODE OP_A (applied by the caller
// when the lines are split over threads: pass ls > 1 and scale afterwards).
template <typename TI, int MODE>
__device__ __forceinline__ float cell2d_sum(const Geom& g, const ViewTables& vt, const ViewHdr& h,
                                            const TI* __restrict__ img_rows, const TI* __restrict__ img_cols,
                                            const int v, const int k, const float cw, const int l0, const int ls) {
    const int Nu = g.Nu;
    const size_t ob = (size_t)v * (Nu + 1) + k;
    const double bA0 = vt.bA[ob], bB0 = vt.bB[ob], bA1 = vt.bA[ob + 1], bB1 = vt.bB[ob + 1];
    const int nlines = h.nlines, npix = h.npix;
    const TI* __restrict__ img = h.use_x ? img_rows : img_cols;
    const float dpixf = (float)h.dpix;
    // arc detector, B^T / Bw^T: the column's upper boundary on the chained
    // walk of a pixel whose first edge lies in this column (every pixel but
    // the band's first); the same on every line
    const bool chain = (MODE == OP_BT || MODE == OP_BWT) && vt.arc;
    const float4* __restrict__ ea = chain ? vt.arc + 2 * (size_t)v * (Nu + 1) : nullptr;
    float d1 = 0.0f;
    if (chain) {
        ArcChain ch;
        ch.start(ea, k, h.keep, (float)g.du);
        d1 = ch.next_exact(h, ea, k + 1);
        if (k + 1 == Nu) d1 = fminf(d1, 0.0f);
    }
    float acc = 0.0f;
    for (int L = l0; L < nlines; L += ls) {
        const double pk = fma(bB0, (double)L, bA0);
        const double pk1 = fma(bB1, (double)L, bA1);
        const int pa = max((int)floor(pk), 0);
        const int pb = min((int)ceil(pk1) - 1, npix - 1);
        if (pa > pb) continue;
        float lf;
        if (MODE == OP_A) lf = __fdividef(dpixf, (float)fma(h.q1, (double)L, h.q0));
        else lf = cw;
        const TI* __restrict__ line = img + (size_t)L * npix;
        // boundaries relative to the first pixel, so FP32 keeps them exact
        float u0 = (float)(pk - (double)pa), u1 = (float)(pk1 - (double)pa);
        float u1b = u1;  // upper boundary for the band's later pixels
        if (chain) {
            const float qd = (float)(fma(h.q1, (double)L, h.q0) / h.dpix);
            u1b = fmaf(d1, qd, u1);
            u1 = u1b;
            if (k > 0 && pk > (double)pa)
                arc_first_pixel_bounds(g, vt, h, ea, v, k, L, pa, pk, pk1, qd, u0, u1);
        }
        for (int pp = pa; pp <= pb; ++pp) {
            const float o = (float)(pp - pa);
            float w = (fminf(o + 1.0f, pp == pa ? u1 : u1b) - fmaxf(o, u0)) * lf;
            if (MODE == OP_BWT) {
                float px, py;
                pixel_center(g, h, L, pp, px, py);
                w *= fbp_weight(g, h, px, py);
            }
            acc = fmaf(w, ld(line + XR_BOUND(pp, 0, npix - 1)), acc);
        }
    }
    if (MODE == OP_A && ls == 1) acc *= vt.colE[(size_t)v * Nu + k];
    return acc;
}

// Voxel gather, 2D: one thread per pixel, sweeping the views.
template <typename TI, typename TO, int MODE>
__global__ void __launch_bounds__(256)
vox_gather2d_kernel(const Geom g, const ViewTables vt, const TI* __restrict__ sino, TO* __restrict__ img,
                    const int nview, const float cw, const float oscale) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int b = blockIdx.z;
    if (ix >= g.W || iy >= g.H) return;
    const float acc = pix2d_sum<TI, MODE>(g, vt, sino + (size_t)b * nview * g.Nu, ix, iy, cw, 0, nview, 1);
    st(img + ((size_t)b * g.H + iy) * g.W + ix, acc * oscale);
}

// Pixel (ix, iy): the 2D DD backprojection sum over views v = v0, v0 + vs, ...
// < v1 of the sinogram sinob [nview][Nu].
template <typename TI, int MODE>
__device__ __forceinline__ float pix2d_sum(const Geom& g, const ViewTables& vt, const TI* __restrict__ sinob,
                                           const int ix, const int iy, const float cw, const int v0,
                                           const int v1, const int vs) {
    const int Nu = g.Nu;
    // This pixel's edges and centre in world coordinates (the values
    // line_point and pixel_center give), hoisted out of the view loop.
    const float dxf = (float)g.dx, dyf = (float)g.dy;
    const float xa_x = (float)(-0.5 * g.W * g.dx + g.shx) + (float)ix * dxf;   // x-axis views: x edges
    const float yc_x = (float)((0.5 * g.H - iy - 0.5) * g.dy + g.shy);          //   and line centre
    const float xc_y = (float)((ix - 0.5 * g.W + 0.5) * g.dx + g.shx);          // y-axis views: line centre
    const float ya_y = (float)(-0.5 * g.H * g.dy + g.shy) + (float)(g.H - 1 - iy) * dyf;  //   and y edges
    const float pcx = (float)((ix - 0.5 * g.W + 0.5) * g.dx + g.shx);  // pixel centre
    const float pcy = (float)((0.5 * g.H - iy - 0.5) * g.dy + g.shy);
    const float sodf = (float)g.sod, shuf = (float)g.shu, inv_du = (float)(1.0 / g.du);
    const float inv_dx = (float)(1.0 / g.dx), inv_dy = (float)(1.0 / g.dy);
    // column bracket margin: half a column, plus the arc guess's angle error
    const float margin = 0.5f + (g.type == GEO_ARC ? XR_GUESS_ATAN_ERR * inv_du : 0.0f);
    float acc = 0.0f;
    for (int v = v0; v < v1; v += vs) {
        const ViewHdr& h = vt.hdr[v];
        int L, p;
        float xa, ya, xb, yb;
        if (h.use_x) {
            L = iy; p = ix;
            xa = xa_x; xb = xa_x + dxf; ya = yb = yc_x;
        } else {
            L = ix; p = g.H - 1 - iy;
            xa = xb = xc_y; ya = ya_y; yb = ya_y + dyf;
        }
        float lf;
        if (MODE == OP_AT) {
            lf = __fdividef((float)h.dpix, (float)fma(h.q1, (double)L, h.q0));
        } else {
            lf = cw;
            if (MODE == OP_BW) lf *= fbp_weight(g, h, pcx, pcy);
        }
        // FP32 column guess (brackets the overlapped columns; the overlaps
        // themselves come from the FP64 boundary tables)
        const float sf = (float)h.s, cf = (float)h.c;
        float kf0, kf1;
        if (g.type == GEO_FLAT) {
            kf0 = (__fdividef(sodf * (xa * cf + ya * sf), sodf + xa * sf - ya * cf) - shuf) * inv_du;
            kf1 = (__fdividef(sodf * (xb * cf + yb * sf), sodf + xb * sf - yb * cf) - shuf) * inv_du;
        } else if (g.type == GEO_ARC) {
            // One guess, at the pixel centre, and a bound on the footprint's
            // half-width: the segment between the pixel's edges on this line
            // (half-length a) seen from the source at distance r from its
            // centre spans at most asin(a / r) <= a / (r - a) rad on each
            // side.  The bracket may take a column more than the edges'
            // own guesses would; the walk skips it.
            const float dcx = h.dcx, dcy = h.dcy;
            const float ex = pcx - (float)h.sx, ey = pcy - (float)h.sy;
            const float kc = guess_atan2f(dcx * ey - dcy * ex, dcx * ex + dcy * ey) * inv_du;
            const float a = 0.5f * (h.use_x ? dxf : dyf);
            const float r2 = fmaf(ex, ex, ey * ey);
            const float r = r2 * rsqrtf(r2);
            const float hw = __fdividef(a, fmaxf(r - a, a)) * inv_du * 1.001f;
            kf0 = kc - hw;
            kf1 = kc + hw;
        } else {
            kf0 = (xa * cf + ya * sf - shuf) * inv_du;
            kf1 = (xb * cf + yb * sf - shuf) * inv_du;
        }
        if (h.keep) { kf0 += 0.5f * Nu; kf1 += 0.5f * Nu; }
        else { kf0 = 0.5f * Nu - kf0; kf1 = 0.5f * Nu - kf1; }
        const float lo = fmaxf(fminf(fminf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const float hi = fmaxf(fminf(fmaxf(kf0, kf1), (float)Nu + 2.0f), -2.0f);
        const int ka = max(0, (int)floorf(lo - margin));
        const int kb = min(Nu - 1, (int)floorf(hi + margin));
        if (ka > kb) continue;
        const double* __restrict__ bA = vt.bA + (size_t)v * (Nu + 1);
        const double* __restrict__ bB = vt.bB + (size_t)v * (Nu + 1);
        const TI* __restrict__ sv = sinob + (size_t)v * Nu;
        const double dp = (double)p, dL = (double)L;
        if (MODE != OP_AT && vt.arc) {
            // arc detector: the pixel's columns walked with chained angles.
            // Boundary ka relative to the pixel in FP64, the next direct
            // boundaries (pd) by adding the columns' widths on this line in
            // FP32, which the walk's arc entries carry.
            const float4* __restrict__ ea = vt.arc + 2 * (size_t)v * (Nu + 1);
            const float Lf = (float)L;
            const float qd = (float)fma(h.q1, dL, h.q0) * (h.use_x ? inv_dx : inv_dy);  // pixels per axis unit
            auto width = [&](int j) { const float4 a = ea[2 * j]; return fmaf(a.w, Lf, a.z); };
            int k = ka;
            float pkl = (float)(fma(bB[k], dL, bA[k]) - dp);
            float pd = pkl + width(k + 1);
            while (!(pd > 0.0f) && k < kb) {
                ++k;
                pkl = pd;
                pd += width(k + 1);
            }
            ArcChain ch;
            ch.start(ea, k, h.keep, (float)g.du);
            float d = ch.next_linear(ea, k + 1);
            if (k + 1 == Nu) d = fminf(d, 0.0f);  // the detector's end
            float pk1 = fmaf(d, qd, pd);
            for (;;) {
                const float wd = fminf(1.0f, pk1) - fmaxf(0.0f, pkl);
                if (wd > 0.0f) {
                    const int col = h.keep ? k : Nu - 1 - k;
                    acc = fmaf(wd * lf, ld(sv + XR_BOUND(col, 0, Nu - 1)), acc);
                }
                if (++k > kb) break;
                pkl = pk1;
                if (pkl >= 1.0f) break;
                float w;
                d = ch.next_linear(ea, k + 1, Lf, w);
                if (k + 1 == Nu) d = fminf(d, 0.0f);
                pd += w;
                pk1 = fmaf(d, qd, pd);
            }
            continue;
        }
        // boundaries relative to the pixel (pixel units)
        float pkl = (float)(fma(bB[ka], dL, bA[ka]) - dp);
        for (int k = ka; k <= kb; ++k) {
            const float pk1 = (float)(fma(bB[k + 1], dL, bA[k + 1]) - dp);
            const float wd = fminf(1.0f, pk1) - fmaxf(0.0f, pkl);
            pkl = pk1;
            if (!(wd > 0.0f)) continue;
            float w = wd * lf;
            if (MODE == OP_AT) w *= vt.colE[(size_t)v * Nu + k];
            const int col = h.keep ? k : Nu - 1 - k;
            acc = fmaf(w, ld(sv + XR_BOUND(col, 0, Nu - 1)), acc);
        }
    }
    return acc;
}

// -------------------------------------------------------------- FBP filter

// out[row, i] = sum_j x[row, j] * filt[j - i + Nu - 1], x = in * cosw * parker.
// A CTA takes `rpc` rows at a time; `tpr` threads per row, each producing 8
// consecutive outputs.  The inner loop runs over blocks of 8 inputs (two
// float4 loads of the row, broadcast to the warp) against a 15-tap register
// window of the filter that advances 8 taps per block: 64 FMAs per 10 shared
// loads.  Taps and rows are zero-padded in shared memory, so the loop has no
// bounds checks.  Neighbouring lanes' windows start 8 taps apart, so the taps
// are stored with one padding float after every 32 (tap i at i + i / 32):
// lanes 4 apart then fall one bank apart instead of on the same bank.
constexpr int XR_FILT_PAD = 32;  // zero taps on each side of the filter

__host__ __device__ inline int filt_row_pitch(int Nu) { return (Nu + 7) / 8 * 8 + 8; }
__host__ __device__ inline int filt_taps_len(int Nu) { return 2 * ((Nu + 7) / 8 * 8) + 2 * XR_FILT_PAD + 16; }
// shared-memory floats holding filt_taps_len taps in the padded layout
__host__ __device__ inline int filt_taps_smem(int Nu) { const int n = filt_taps_len(Nu); return n + n / 32 + 1; }
__device__ __forceinline__ int tap_pos(int i) { return i + (i >> 5); }

// Row source of the filter: a stored sinogram row times the cosine and
// Parker weights.
template <typename TI>
struct SinoRows {
    const TI* in;
    const float* cosw;
    const float* parker;
    int Nu, nview, rows_per_view;
    __device__ __forceinline__ float operator()(int row, int j) const {
        float val = ld(in + (size_t)row * Nu + j);
        if (cosw) val *= cosw[j];
        if (parker) val *= parker[(size_t)((row / rows_per_view) % nview) * Nu + j];
        return val;
    }
};

template <typename Rows, int OUTS>
__global__ void __launch_bounds__(256)
fbp_filter_kernel(const Rows src, float* __restrict__ out, const int nrows, const int Nu,
                  const float* __restrict__ filt, const int tpr, const int rpc) {
    static_assert(OUTS == 8, "the register window below is written for 8 outputs per thread");
    extern __shared__ __align__(16) float smem[];
    const int nf = 2 * Nu - 1;
    const int ntap = filt_taps_len(Nu);
    const int pitch = filt_row_pitch(Nu);
    float* fp = smem;                               // fp[tap_pos(XR_FILT_PAD + m)] = filt[m]
    float* xs = smem + (filt_taps_smem(Nu) + 3) / 4 * 4;  // rpc rows of `pitch` floats
    for (int i = threadIdx.x; i < ntap; i += blockDim.x) {
        const int m = i - XR_FILT_PAD;
        fp[tap_pos(i)] = (m >= 0 && m < nf) ? filt[m] : 0.0f;
    }
    const int r = threadIdx.x / tpr, tl = threadIdx.x - r * tpr;
    for (int row0 = blockIdx.x * rpc; row0 < nrows; row0 += gridDim.x * rpc) {
        __syncthreads();
        for (int e = threadIdx.x; e < rpc * pitch; e += blockDim.x) {
            const int rr = e / pitch, j = e - rr * pitch;
            const int row = row0 + rr;
            xs[e] = (j < Nu && row < nrows) ? src(row, j) : 0.0f;
        }
        __syncthreads();
        const int row = row0 + r;
        if (r >= rpc || row >= nrows) continue;
        const float* xr = xs + r * pitch;
        for (int i0 = tl * OUTS; i0 < Nu; i0 += tpr * OUTS) {
            // out[i0 + t] = sum_j x[j] fb[j - t],  fb[m] = filt[m + Nu - 1 - i0]
            const int fb0 = XR_FILT_PAD + (Nu - 1 - i0);  // tap index of fb[0]
            float acc[OUTS];
#pragma unroll
            for (int t = 0; t < OUTS; ++t) acc[t] = 0.0f;
            float w[15];  // w[k] = fb[jb - 7 + k]
#pragma unroll
            for (int k = 0; k < 7; ++k) w[k] = fp[tap_pos(fb0 + k - 7)];
            for (int jb = 0; jb < Nu; jb += 8) {
                const float4 xa = *reinterpret_cast<const float4*>(xr + jb);
                const float4 xb = *reinterpret_cast<const float4*>(xr + jb + 4);
                const float x8[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
#pragma unroll
                for (int k = 0; k < 8; ++k) w[7 + k] = fp[tap_pos(fb0 + jb + k)];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj)
#pragma unroll
                    for (int t = 0; t < OUTS; ++t) acc[t] = fmaf(x8[jj], w[jj - t + 7], acc[t]);
#pragma unroll
                for (int k = 0; k < 7; ++k) w[k] = w[k + 8];
            }
#pragma unroll
            for (int t = 0; t < OUTS; ++t)
                if (i0 + t < Nu) out[(size_t)row * Nu + i0 + t] = acc[t];
        }
    }
}

}  // namespace xr
