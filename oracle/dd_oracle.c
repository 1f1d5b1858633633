/*
 * dd_oracle.c -- FP64 CPU restatement of XRecon's distance-driven (DD)
 * operators.  TEST INFRASTRUCTURE ONLY: the product never links, loads or
 * calls this file; tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it as the reference result to compare against.
 *
 * What it restates (paths relative to the XRecon project root):
 *   geometry conventions   include/types.h:35-119, include/xrmath.h:8-226
 *   2D projection A        src/cpu/system_matrix2d.cpp:96-365
 *                          (matrix_parallel / matrix_fanflat / matrix_fanarc)
 *   2D A^T                 src/cpu/forward2d.cpp:80-112 (adjoint of A)
 *   2D B, Bw               src/cpu/backward2d.cpp:30-250
 *   2D B^T, Bw^T           src/cpu/backward2d.cpp:258-473
 *   3D cone A, A^T         src/cpu/forward3d.cpp:299-585
 *   3D cone B, Bw, B^T     include/cpu3d_common.h:48-202,
 *                          src/cpu/backward3d.cpp:10-135
 *   3D parallel            src/cpu/forward3d.cpp:37-181 (B = A^T, B^T = A)
 *
 * Formulation.  For every view the reference maps detector-cell boundaries
 * and voxel boundaries onto one common axis (the x axis when cos^2 > 1/2,
 * else the y axis) and, in 3D, maps z boundaries onto that axis' plane with
 * the magnification of the detector column centre (cells) and of the voxel
 * line centre (voxels).  Every operator is the same overlap kernel
 *     K[cell, voxel] = |pixel_axis cap column_axis| * |voxel_z cap row_z|
 * with a diagonal scale on one side:
 *     A   = S_cell K,        A^T = K^T S_cell,
 *     B^T = K T_vox,         B   = T_vox K^T       (Bw: T_vox includes w).
 * The reference evaluates K with sequential merges in float32; this file
 * evaluates the identical overlaps with a two-pointer merge in double
 * precision.  The decisions the reference takes in float (which axis, which
 * detector traversal order) are taken from float sin/cos of the float angle,
 * as the reference CPU path does (std::sin/std::cos on float).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { GEO_PARALLEL = 0, GEO_FLAT = 1, GEO_ARC = 2 };
enum { OP_A = 0, OP_AT = 1, OP_B = 2, OP_BT = 3, OP_BW = 4, OP_BWT = 5 };

typedef struct {
    int use_x;   /* common axis is x (xrmath.h usage: cos^2 > 0.5) */
    int keep;    /* detector traversed in index order (keep_dim) */
    double beta, s, c;
    double sx, sy;        /* source position, xrmath.h:116-123 */
    double spar, sperp;   /* source coordinate along / across the axis */
} view_t;

static view_t make_view(float ang, double sod)
{
    view_t v;
    const float cf = cosf(ang);
    const float sf = sinf(ang);
    v.use_x = (cf * cf > 0.5f);
    v.keep = v.use_x ? (cf >= 0.0f) : (sf >= 0.0f);
    v.beta = (double)ang;
    v.s = sin(v.beta);
    v.c = cos(v.beta);
    v.sx = -v.s * sod;
    v.sy = v.c * sod;
    v.spar = v.use_x ? v.sx : v.sy;
    v.sperp = v.use_x ? v.sy : v.sx;
    return v;
}

/* Signed boundary offset of traversal boundary k (k may be fractional for
 * cell centres): xrmath.h / forward3d.cpp:236-238 use (k - Nu/2) when the
 * detector is kept in order and (Nu/2 - k) when it is reversed. */
static double sigma(const view_t* v, double k, int nu)
{
    return v->keep ? (k - 0.5 * nu) : (0.5 * nu - k);
}

/* map2x / map2y of xrmath.h:8-22: intercept of the ray source->point with
 * the common axis. */
static double map_point(const view_t* v, double px, double py)
{
    if (v->use_x) return (v->sx * py - v->sy * px) / (py - v->sy);
    return (v->sy * px - v->sx * py) / (px - v->sx);
}

/* map2x / map2y for a ray leaving the source at angle a (xrmath.h:24-38). */
static double map_angle(const view_t* v, double a)
{
    if (v->use_x) return v->sx + v->sy * tan(a);
    return v->sy + v->sx / tan(a);
}

/* Arc boundary and column-centre angles as the reference forms them: in
 * float32 with every operation rounded, (k - Nu/2) du + shift_u + beta for a
 * detector kept in order and (Nu/2 - k) du + shift_u + beta for a reversed
 * one (forward3d.cpp:271-297, system_matrix2d.cpp:280-283).  The rounding of
 * the last sum (a quantum of 4.8e-7 rad at |beta| ~ 2 pi) moves a boundary by
 * up to 3e-4 of a detector cell, so the operator follows it; everything
 * after the angle is FP64.  xo_set_arc_exact(1) switches to the exact angle. */
static int g_arc_exact = 0;

void xo_set_arc_exact(int on) { g_arc_exact = on; }

/* Axis position of an arc boundary angle as the reference maps it: in
 * float32, src.x + src.y tanf(a) (x axis) or src.y + src.x / tanf(a) (y axis)
 * with the float source (-sinf(b) SOD, cosf(b) SOD) (xrmath.h:24-38,
 * :116-123).  The sum cancels: its rounding, about ulp(|src|), is up to 1e-4
 * of a column near the 45-degree views and the voxel-driven coefficients
 * scale with it.  g_tan_cr = 1 takes tan correctly rounded to float instead
 * of the C library's tanf (which is not always), and the voxel-driven B and Bw
 * take the chained boundaries linearised around the direct ones
 * (chain_overlaps): the CUDA path's arithmetic. */
static int g_tan_cr = 0;

void xo_set_tan_rounding(int correctly_rounded) { g_tan_cr = correctly_rounded; }

static double map_angle_f(const view_t* v, float a, double sod)
{
    const float b = (float)v->beta, R = (float)sod;
    volatile float sx = -sinf(b) * R, sy = cosf(b) * R;
    volatile float t = g_tan_cr ? (float)tan((double)a) : tanf(a);
    volatile float r;
    if (v->use_x) { volatile float m = sy * t; r = sx + m; }
    else          { volatile float q = sx / t; r = sy + q; }
    return (double)r;
}

static double arc_angle(const view_t* v, double k, int nu, double du, double shu)
{
    if (g_arc_exact) return sigma(v, k, nu) * du + shu + v->beta;
    volatile float s = v->keep ? ((float)k - (float)nu * 0.5f) : ((float)nu * 0.5f - (float)k);
    volatile float a = s * (float)du;
    a = a + (float)shu;
    a = a + (float)v->beta;
    return (double)a;
}

/* Column overlaps of the pixels of one line for the voxel-driven arc
 * operators (B, Bw and their transposes).  The reference walks each voxel's
 * columns with boundary angles chained in float32 from the voxel's first
 * column (include/cpu3d_common.h:150-196, src/cpu/backward2d.cpp:119-157):
 * the first angle is that column's (lower, kept detector) or the next
 * column's plus du (reversed detector), each further one is the previous
 * plus or minus du, rounded.  The overlaps with the pixel [X[p], X[p+1]]
 * follow those angles; the column's z magnification uses the mid angle
 * 0.5 (a + a_next) of the pair.  Entries go to (ia, ib, len, cang) like
 * overlaps(); D holds the boundaries of arc_angle (the detector ends). */
static int chain_overlaps(const view_t* v, const double* X, int npix, const double* D, int nu,
                          double du, double shu, double sod, int linear, int* ia, int* ib, double* len,
                          double* cang)
{
    int n = 0;
    const float duf = (float)du;
    for (int p = 0; p < npix; ++p) {
        double b0 = X[p] > D[0] ? X[p] : D[0];
        const double b1 = X[p + 1] < D[nu] ? X[p + 1] : D[nu];
        if (!(b0 < b1)) continue;
        int k = 0;
        while (k < nu - 1 && D[k + 1] <= b0) ++k;
        volatile float t;
        if (v->keep) {
            t = (float)arc_angle(v, k, nu, du, shu);
        } else {
            volatile float t1 = (float)arc_angle(v, k + 1, nu, du, shu);
            t = t1 + duf;
        }
        while (b0 < b1 && k < nu) {
            volatile float tn = v->keep ? t + duf : t - duf;
            double Dn = g_arc_exact ? map_angle(v, (double)tn) : map_angle_f(v, tn, sod);
            if (linear && !g_arc_exact) {
                /* direct boundary k + 1 and the derivative of the axis map there */
                const double td = arc_angle(v, k + 1, nu, du, shu);
                const double Dd = map_angle_f(v, (float)td, sod);
                const double tt = tan(td);
                const double dDdt = v->use_x ? v->sy * (1.0 + tt * tt) : -v->sx * (1.0 + tt * tt) / (tt * tt);
                Dn = Dd + ((double)tn - td) * dDdt;
            }
            const double nb = b1 < Dn ? b1 : Dn;
            const double ov = nb - b0;
            if (ov > 0.0) {
                volatile float sum = t + tn;
                ia[n] = p; ib[n] = k; len[n] = ov; cang[n] = (double)(0.5f * sum); ++n;
            }
            b0 = ov > 0.0 ? nb : Dn;
            t = tn;
            ++k;
        }
    }
    return n;
}

/* Two-pointer merge of the interval sequences [a_i, a_{i+1}] (i < na) and
 * [b_j, b_{j+1}] (j < nb), both increasing.  Writes the overlapping pairs. */
static int overlaps(const double* a, int na, const double* b, int nb,
                    int* ia, int* ib, double* len)
{
    int i = 0, j = 0, n = 0;
    while (i < na && j < nb) {
        const double lo = a[i] > b[j] ? a[i] : b[j];
        const double hi = a[i + 1] < b[j + 1] ? a[i + 1] : b[j + 1];
        if (hi > lo) { ia[n] = i; ib[n] = j; len[n] = hi - lo; ++n; }
        if (a[i + 1] < b[j + 1]) ++i; else ++j;
    }
    return n;
}

/* ---------------------------------------------------------------- 3D ---- */

typedef struct {
    int W, H, D, Nu, Nv, type;
    double dx, dy, dz, shx, shy, shz;
    double du, dv, shu, shv, sod, sdd;
} geo3_t;

/* Per view: column boundaries on the axis (Nu+1), column-centre z scale
 * (Nu), row boundaries before magnification (Nv+1). */
static void view_columns3d(const geo3_t* g, const view_t* v,
                           double* D, double* M, double* zd)
{
    const double vs = g->sod / g->sdd;
    for (int k = 0; k <= g->Nu; ++k) {
        if (g->type == GEO_FLAT) {
            /* forward3d.cpp:229-243 (virtual detector through isocentre) */
            const double u = (sigma(v, k, g->Nu) * g->du + g->shu) * vs;
            D[k] = map_point(v, u * v->c, u * v->s);
        } else if (g->type == GEO_ARC) {
            /* forward3d.cpp:271-283 */
            const double a = arc_angle(v, k, g->Nu, g->du, g->shu);
            D[k] = g_arc_exact ? map_angle(v, a) : map_angle_f(v, (float)a, g->sod);
        } else {
            /* forward3d.cpp:53-56 (parallel: u / cos or u / sin) */
            const double u = sigma(v, k, g->Nu) * g->du + g->shu;
            D[k] = v->use_x ? u / v->c : u / v->s;
        }
    }
    for (int k = 0; k < g->Nu; ++k) {
        double cx, cy;
        if (g->type == GEO_FLAT) {
            /* forward3d.cpp:258-269 */
            const double u = (sigma(v, k + 0.5, g->Nu) * g->du + g->shu) * vs;
            cx = u * v->c; cy = u * v->s;
        } else if (g->type == GEO_ARC) {
            /* forward3d.cpp:285-297 */
            const double a = arc_angle(v, k + 0.5, g->Nu, g->du, g->shu);
            cx = sin(a) * g->sdd + v->sx; cy = -cos(a) * g->sdd + v->sy;
        } else {
            cx = cy = 0.0;
        }
        if (g->type == GEO_PARALLEL) M[k] = 1.0;
        else M[k] = v->use_x ? v->sy / (v->sy - cy) : v->sx / (v->sx - cx);
    }
    /* forward3d.cpp:318-320: flat rows live on the virtual detector. */
    const double rs = (g->type == GEO_FLAT) ? vs : 1.0;
    for (int r = 0; r <= g->Nv; ++r) zd[r] = ((r - 0.5 * g->Nv) * g->dv + g->shv) * rs;
}

/* Axis boundaries of the pixels of one line and the line's z magnification.
 * Lines are volume rows iy (x axis) or volume columns ix (y axis);
 * forward3d.cpp:372-384 and :432-444. */
static int line_pixels3d(const geo3_t* g, const view_t* v, int line,
                         double* X, double* Mv, double* perp_coord)
{
    if (v->use_x) {
        const double py = (0.5 * g->H - line - 0.5) * g->dy + g->shy;
        const double x0 = -0.5 * g->W * g->dx + g->shx;
        for (int i = 0; i <= g->W; ++i) {
            const double x = x0 + i * g->dx;
            X[i] = (g->type == GEO_PARALLEL) ? (v->s / v->c) * py + x : map_point(v, x, py);
        }
        *Mv = (g->type == GEO_PARALLEL) ? 1.0 : v->sy / (v->sy - py);
        *perp_coord = py;
        return g->W;
    } else {
        const double px = (line - 0.5 * g->W + 0.5) * g->dx + g->shx;
        const double y0 = -0.5 * g->H * g->dy + g->shy;
        for (int i = 0; i <= g->H; ++i) {
            const double y = y0 + i * g->dy;
            X[i] = (g->type == GEO_PARALLEL) ? (v->c / v->s) * px + y : map_point(v, px, y);
        }
        *Mv = (g->type == GEO_PARALLEL) ? 1.0 : v->sx / (v->sx - px);
        *perp_coord = px;
        return g->H;
    }
}

/* Voxel centre coordinates (xrmath.h:163-173; image row 0 is the top). */
static void voxel_xy(const geo3_t* g, int ix, int iy, double* px, double* py)
{
    *px = (ix - 0.5 * g->W + 0.5) * g->dx + g->shx;
    *py = (0.5 * g->H - iy - 0.5) * g->dy + g->shy;
}

/* FBP voxel weight: cone_voxel_weight_flat / _arc (xrmath.h:215-226). */
static double fbp_weight(int type, const view_t* v, double sod, double px, double py)
{
    if (type == GEO_FLAT) {
        const double d = (v->sx * px + v->sy * py) / sod;
        return sod * sod / ((sod - d) * (sod - d));
    }
    if (type == GEO_ARC) {
        const double ex = v->sx - px, ey = v->sy - py;
        return 1.0 / (ex * ex + ey * ey);
    }
    return 1.0;
}

/* Apply one 3D operator.  Layouts: image [nb][D][H][W], sino [nb][V][Nv][Nu].
 * `in` is read, `out` is overwritten. */
int xo_dd3d(int op, const int* ni, const double* fv, const double* fg, int type,
            const double* in, double* out, const float* ang, int nbatch, int nview)
{
    geo3_t g;
    g.W = ni[0]; g.H = ni[1]; g.D = ni[2]; g.Nu = ni[3]; g.Nv = ni[4]; g.type = type;
    g.dx = fv[0]; g.dy = fv[1]; g.dz = fv[2]; g.shx = fv[3]; g.shy = fv[4]; g.shz = fv[5];
    g.du = fg[0]; g.dv = fg[1]; g.shu = fg[2]; g.shv = fg[3]; g.sod = fg[4]; g.sdd = fg[5];
    if (op < 0 || op > 5) return 1;
    if (type == GEO_PARALLEL) {
        /* backward3d.cpp:101-135: parallel B = Bw = A^T and B^T = Bw^T = A. */
        if (op == OP_B || op == OP_BW) op = OP_AT;
        else if (op == OP_BT || op == OP_BWT) op = OP_A;
    }
    const long long nvox = (long long)g.W * g.H * g.D;
    const long long ncell = (long long)g.Nu * g.Nv;
    const int out_is_sino = (op == OP_A || op == OP_BT || op == OP_BWT);
    memset(out, 0, sizeof(double) * (size_t)nbatch *
           (size_t)(out_is_sino ? ncell * nview : nvox));

    const int nline_max = g.W > g.H ? g.W : g.H;
    double* D = malloc(sizeof(double) * (g.Nu + 1));
    double* M = malloc(sizeof(double) * g.Nu);
    double* zd = malloc(sizeof(double) * (g.Nv + 1));
    double* X = malloc(sizeof(double) * (nline_max + 1));
    double* Zv = malloc(sizeof(double) * (g.D + 1));
    double* Zc = malloc(sizeof(double) * (g.Nv + 1));
    const int nxo = nline_max + g.Nu + 2, nzo = g.D + g.Nv + 2;
    int* xa = malloc(sizeof(int) * nxo); int* xb = malloc(sizeof(int) * nxo);
    double* xl = malloc(sizeof(double) * nxo);
    int* za = malloc(sizeof(int) * nzo); int* zb = malloc(sizeof(int) * nzo);
    double* zl = malloc(sizeof(double) * nzo);

    const double z0 = -0.5 * g.D * g.dz + g.shz;
    const double cw = (type == GEO_FLAT) ? g.du * g.sod / g.sdd
                    : (type == GEO_ARC) ? 2.0 * g.sod * tan(0.5 * g.du) : g.du;
    /* voxel-driven arc operators: columns chained per voxel as the reference does */
    const int chain = type == GEO_ARC && !g_arc_exact && op != OP_A && op != OP_AT;
    double* xc = malloc(sizeof(double) * nxo);

    for (int view = 0; view < nview; ++view) {
        const view_t v = make_view(ang[view], g.sod);
        view_columns3d(&g, &v, D, M, zd);
        const double dperp = v.use_x ? g.dy : g.dx;
        const int nlines = v.use_x ? g.H : g.W;
        for (int line = 0; line < nlines; ++line) {
            double Mv, perp;
            const int npix = line_pixels3d(&g, &v, line, X, &Mv, &perp);
            for (int i = 0; i <= g.D; ++i) Zv[i] = Mv * (z0 + i * g.dz);
            const int nx = chain ? chain_overlaps(&v, X, npix, D, g.Nu, g.du, g.shu, g.sod, g_tan_cr && (op == OP_B || op == OP_BW), xa, xb, xl, xc)
                                 : overlaps(X, npix, D, g.Nu, xa, xb, xl);
            for (int e = 0; e < nx; ++e) {
                const int p = xa[e], k = xb[e];
                const int ix = v.use_x ? p : line;
                const int iy = v.use_x ? line : g.H - 1 - p;
                const int col = v.keep ? k : g.Nu - 1 - k;
                double Mk = M[k];
                if (chain) {
                    const double cx = sin(xc[e]) * g.sdd + v.sx, cy = -cos(xc[e]) * g.sdd + v.sy;
                    Mk = v.use_x ? v.sy / (v.sy - cy) : v.sx / (v.sx - cx);
                }
                for (int r = 0; r <= g.Nv; ++r) Zc[r] = Mk * zd[r];
                const int nz = overlaps(Zv, g.D, Zc, g.Nv, za, zb, zl);
                /* voxel-side scale: reference voxel_area = |(X1-X0)(z1-z0)|
                 * (cpu3d_common.h:80) and the FBP weight (:84-85). */
                double tvox = 0.0;
                if (op == OP_B || op == OP_BT || op == OP_BW || op == OP_BWT) {
                    tvox = cw / ((X[p + 1] - X[p]) * Mv * g.dz);
                    if (op == OP_BW || op == OP_BWT) {
                        double px, py;
                        voxel_xy(&g, ix, iy, &px, &py);
                        tvox *= fbp_weight(type, &v, g.sod, px, py);
                    }
                }
                for (int q = 0; q < nz; ++q) {
                    const int iz = za[q], r = zb[q];
                    const double coef = xl[e] * zl[q];
                    double sa = 1.0;
                    if (op == OP_A || op == OP_AT) {
                        if (type == GEO_PARALLEL) {
                            /* forward3d.cpp:58, :98: xy_scale / dv */
                            sa = dperp / (g.du * g.dv);
                        } else {
                            /* forward3d.cpp:331-343 */
                            const double dD = D[k + 1] - D[k];
                            const double dZ = Zc[r + 1] - Zc[r];
                            const double a = 0.5 * (D[k + 1] + D[k]) - v.spar;
                            const double b = 0.5 * (Zc[r + 1] + Zc[r]);
                            const double cosw = fabs(v.sperp) / sqrt(a * a + b * b + v.sperp * v.sperp);
                            sa = dperp / (dD * dZ * cosw);
                        }
                    }
                    for (int bt = 0; bt < nbatch; ++bt) {
                        const long long vi = ((long long)(bt * g.D + iz) * g.H + iy) * g.W + ix;
                        const long long ci = (((long long)bt * nview + view) * g.Nv + r) * g.Nu + col;
                        switch (op) {
                        case OP_A:   out[ci] += coef * sa * in[vi]; break;
                        case OP_AT:  out[vi] += coef * sa * in[ci]; break;
                        case OP_B:
                        case OP_BW:  out[vi] += coef * tvox * in[ci]; break;
                        default:     out[ci] += coef * tvox * in[vi]; break;
                        }
                    }
                }
            }
        }
    }
    free(D); free(M); free(zd); free(X); free(Zv); free(Zc);
    free(xa); free(xb); free(xl); free(za); free(zb); free(zl); free(xc);
    return 0;
}

/* ---------------------------------------------------------------- 2D ---- */

/* 2D geometry values are the packed ones of the reference options tensor
 * (projector.py:97-110): du and shu are already "effective" (flat: scaled to
 * the isocentre; arc: angular). */
int xo_dd2d(int op, const int* ni, const double* fv, const double* fg, int type,
            const double* in, double* out, const float* ang, int nbatch, int nview)
{
    const int W = ni[0], H = ni[1], Nu = ni[2];
    const double dx = fv[0], dy = fv[1], shx = fv[2], shy = fv[3];
    const double du = fg[0], shu = fg[1], sod = fg[2];
    if (op < 0 || op > 5) return 1;
    const int out_is_sino = (op == OP_A || op == OP_BT || op == OP_BWT);
    memset(out, 0, sizeof(double) * (size_t)nbatch *
           (size_t)(out_is_sino ? (long long)Nu * nview : (long long)W * H));
    const int nline_max = W > H ? W : H;
    double* D = malloc(sizeof(double) * (Nu + 1));
    double* X = malloc(sizeof(double) * (nline_max + 1));
    const int nxo = nline_max + Nu + 2;
    int* xa = malloc(sizeof(int) * nxo); int* xb = malloc(sizeof(int) * nxo);
    double* xl = malloc(sizeof(double) * nxo);
    /* B column width: backward2d.cpp:87 (flat du), :109 (arc 2 SOD tan(du/2)),
     * :185 (parallel du / pixel). */
    const double cw = (type == GEO_ARC) ? 2.0 * sod * tan(0.5 * du) : du;
    const int chain = type == GEO_ARC && !g_arc_exact && op != OP_A && op != OP_AT;
    double* xc = malloc(sizeof(double) * nxo);

    for (int view = 0; view < nview; ++view) {
        const view_t v = make_view(ang[view], sod);
        for (int k = 0; k <= Nu; ++k) {
            const double sg = sigma(&v, k, Nu);
            if (type == GEO_FLAT) {
                /* system_matrix2d.cpp:185-189 */
                const double u = sg * du + shu;
                D[k] = map_point(&v, u * v.c, u * v.s);
            } else if (type == GEO_ARC) {
                /* system_matrix2d.cpp:280-283 */
                const double a = arc_angle(&v, k, Nu, du, shu);
                D[k] = g_arc_exact ? map_angle(&v, a) : map_angle_f(&v, (float)a, sod);
            } else {
                /* system_matrix2d.cpp:104-107 */
                const double u = sg * du + shu;
                D[k] = v.use_x ? u / v.c : u / v.s;
            }
        }
        const double dperp = v.use_x ? dy : dx;
        const int nlines = v.use_x ? H : W;
        for (int line = 0; line < nlines; ++line) {
            int npix;
            if (v.use_x) {
                const double py = (0.5 * H - line - 0.5) * dy + shy;
                const double x0 = -0.5 * W * dx + shx;
                for (int i = 0; i <= W; ++i)
                    X[i] = (type == GEO_PARALLEL) ? (v.s / v.c) * py + x0 + i * dx
                                                   : map_point(&v, x0 + i * dx, py);
                npix = W;
            } else {
                const double px = (line - 0.5 * W + 0.5) * dx + shx;
                const double y0 = -0.5 * H * dy + shy;
                for (int i = 0; i <= H; ++i)
                    X[i] = (type == GEO_PARALLEL) ? (v.c / v.s) * px + y0 + i * dy
                                                   : map_point(&v, px, y0 + i * dy);
                npix = H;
            }
            const int nx = chain ? chain_overlaps(&v, X, npix, D, Nu, du, shu, sod, g_tan_cr && (op == OP_B || op == OP_BW), xa, xb, xl, xc)
                                 : overlaps(X, npix, D, Nu, xa, xb, xl);
            for (int e = 0; e < nx; ++e) {
                const int p = xa[e], k = xb[e];
                const int ix = v.use_x ? p : line;
                const int iy = v.use_x ? line : H - 1 - p;
                const int col = v.keep ? k : Nu - 1 - k;
                double scale;
                if (op == OP_A || op == OP_AT) {
                    if (type == GEO_PARALLEL) {
                        scale = dperp / du;            /* system_matrix2d.cpp:109 */
                    } else {
                        /* system_matrix2d.cpp:213, :251 (cos_weight_x/y) */
                        const double a = 0.5 * (D[k + 1] + D[k]) - v.spar;
                        const double cosw = fabs(v.sperp) / sqrt(a * a + v.sperp * v.sperp);
                        scale = dperp / ((D[k + 1] - D[k]) * cosw);
                    }
                } else {
                    scale = cw / (X[p + 1] - X[p]);
                    if ((op == OP_BW || op == OP_BWT) && type != GEO_PARALLEL) {
                        const double px = (ix - 0.5 * W + 0.5) * dx + shx;
                        const double py = (0.5 * H - iy - 0.5) * dy + shy;
                        scale *= fbp_weight(type, &v, sod, px, py);
                    }
                }
                const double coef = xl[e] * scale;
                for (int bt = 0; bt < nbatch; ++bt) {
                    const long long vi = ((long long)bt * H + iy) * W + ix;
                    const long long ci = ((long long)bt * nview + view) * Nu + col;
                    if (op == OP_A || op == OP_BT || op == OP_BWT) out[ci] += coef * in[vi];
                    else out[vi] += coef * in[ci];
                }
            }
        }
    }
    free(D); free(X); free(xa); free(xb); free(xl); free(xc);
    return 0;
}

/* ----------------------------------------------------------- helical ---- */
/*
 * Helical cone-beam operators with an arc detector (XRecon
 * src/kernels/helical_arc3d.cu, bound at src/api/torch_binding.cpp:525-612,
 * Python xrecon/projector/projector3d.py:289-576).
 *
 * A, A^T, B, B^T (helical_arc3d.cu:364-1111, :1507-1761) are the cone-arc DD
 * operators above with per-view geometry taken from source_pos [4][V] =
 * (source_z, shift_radius, shift_angle, shift_z), helical_arc3d.cu:382-395:
 *     sod' = SOD + sr, sdd' = SDD + sr, du' = du SDD / sdd',
 *     shu' = shu SDD / sdd' - sa (sdd' - sod') / sdd',
 *     source at angle beta + sa (float sum), column angles sg du' + shu' + beta,
 *     source z = source_z + shift_z, detector rows at
 *     (r - Nv/2) dv + source_z + shv,
 * all z measured from the source z.  Two details follow the reference:
 *   - A's cell cosine (triangle_cosine, helical_arc3d.cu:432) takes the mean
 *     row position on the axis plane WITHOUT subtracting the source z
 *     (det_row_axis carries "+ src_z");
 *   - B's column width is sod' du' (helical_arc3d.cu:896).
 * The per-view scalars are formed in float as the reference forms them; the
 * overlaps are evaluated in double as in xo_dd3d.
 *
 * Bw and Bw^T (helical_arc3d.cu:1112-1505) weight every (voxel, view) pair
 * of the voxel's view window with a redundancy weight and normalise per
 * voxel; the weights are restated below in float with the reference's
 * operation order, the DD footprint in double.
 */

#define XO_PI_F 3.14159265358979323846f

typedef struct {
    int view_mode, weight_mode;
    float view_turns, halfscan_coef, tang_k, tang_blend;
    /* pin aid: take the window length's quotient span/|dbeta| one float ulp
     * up before ceil(), as the reference's --use_fast_math division turned
     * out to do at an exact integer quotient (tests/golden/helical_ref_*) */
    int window_quotient_up;
} hopt_t;

typedef struct {
    geo3_t g;        /* sod, sdd, du, shu of this view */
    view_t v;        /* source at float(beta + shift_angle), radius sod' */
    double zsrc;     /* source z */
    double zrow0;    /* lower boundary of detector row 0, relative to zsrc */
    double cwB;      /* B / B^T column width sod' du' */
} hview_t;

static void helical_view(const geo3_t* g0, const float* ang, const float* sp, int nview, int view, hview_t* h)
{
    const float zs = sp[view], sr = sp[nview + view], sa = sp[2 * nview + view], szs = sp[3 * nview + view];
    const float SOD = (float)g0->sod, SDD = (float)g0->sdd, du0 = (float)g0->du, shu0 = (float)g0->shu;
    const float sod = SOD + sr;
    const float sdd = SDD + sr;
    const float du = du0 * SDD / sdd;
    const float shu = shu0 * SDD / sdd - sa * (sdd - sod) / sdd;
    const float beta = ang[view] + sa;
    const float zsrc = zs + szs;
    h->g = *g0;
    h->g.sod = sod;
    h->g.sdd = sdd;
    h->g.du = du;
    /* column angle sg du' + shu' + beta_unshifted, written relative to the
     * source angle the header carries */
    h->g.shu = (double)shu + ((double)ang[view] - (double)beta);
    h->v = make_view(beta, sod);
    h->zsrc = zsrc;
    h->zrow0 = -0.5 * g0->Nv * g0->dv + (double)zs + g0->shv - (double)zsrc;
    h->cwB = (double)(sod * du);
}

/* ---- weights, float, helical_arc3d.cu:8-336 ---- */

static float hw_clamp_unit(float x) { return fminf(1.0f, fmaxf(0.0f, x)); }

static float hw_smooth_step(float x)
{
    x = hw_clamp_unit(x);
    return 0.5f * (1.0f - cosf(XO_PI_F * x));
}

static float hw_window_quality(float beta, float bs, float be, float gamma, float gmax)
{
    const float lo = fminf(bs, be), hi = fmaxf(bs, be);
    if (beta < lo || beta > hi) return 0.0f;
    const float gc = fminf(fmaxf(gamma, -gmax), gmax);
    const float lw = fmaxf(1.0e-6f, 2.0f * (gmax - gc));
    const float rw = fmaxf(1.0e-6f, 2.0f * (gmax + gc));
    if (beta < lo + lw) return hw_smooth_step((beta - lo) / lw);
    if (beta > hi - rw) return hw_smooth_step((hi - beta) / rw);
    return 1.0f;
}

static float hw_center_turn(float beta, float bc, float bs, float be, float db)
{
    const float lo = fminf(bs, be), hi = fmaxf(bs, be);
    if (beta < lo || beta > hi) return 0.0f;
    const float adb = fmaxf(fabsf(db), 1.0e-6f);
    const float half = 0.5f * (hi - lo);
    const float dist = fabsf(beta - bc);
    const float crad = fminf(XO_PI_F, half);
    if (dist <= crad) return 1.0f;
    const float ow = fmaxf(half - crad, 4.0f * adb);
    return hw_smooth_step((half - dist) / ow);
}

static float hw_source_z_at(float beta, const float* ang, const float* zsrc, int nview)
{
    if (nview <= 1) return zsrc[0];
    const float a0 = ang[0], a1 = ang[nview - 1];
    const float range = a1 - a0;
    if (fabsf(range) <= 1.0e-6f) return zsrc[0];
    const float dzdb = (zsrc[nview - 1] - zsrc[0]) / range;
    return zsrc[0] + (beta - a0) * dzdb;
}

static float hw_edge_taper(float beta, float bc, float bs, float be, float db)
{
    const float lo = fminf(bs, be), hi = fmaxf(bs, be);
    if (beta < lo || beta > hi) return 0.0f;
    const float span = hi - lo, half = 0.5f * span;
    if (span <= XO_PI_F + 8.0f * fabsf(db)) return 1.0f;
    const float crad = fminf(XO_PI_F, half);
    const float dist = fabsf(beta - bc);
    if (dist <= crad) return 1.0f;
    const float ew = fmaxf(half - crad, 4.0f * fabsf(db));
    return hw_smooth_step((half - dist) / ew);
}

static float hw_center_beta(float pz, const float* ang, const float* zsrc, int vs, int ve, int nview)
{
    const float bs = ang[vs], be = ang[ve];
    if (nview <= 1) return 0.5f * (bs + be);
    const float a0 = ang[0], a1 = ang[nview - 1], z0 = zsrc[0], z1 = zsrc[nview - 1];
    const float range = a1 - a0;
    const float dzdb = (fabsf(range) > 1.0e-6f) ? (z1 - z0) / range : 0.0f;
    if (fabsf(dzdb) <= 1.0e-8f) return 0.5f * (bs + be);
    const float beta = a0 + (pz - z0) / dzdb;
    return fminf(fmaxf(beta, fminf(bs, be)), fmaxf(bs, be));
}

/* helical_arc3d.cu:141-210 */
static void hw_view_window(float pz, const float* ang, const float* zsrc, const geo3_t* g, const hopt_t* o,
                           int nview, int* vs, int* ve)
{
    if (nview <= 1) { *vs = 0; *ve = 0; return; }
    const float a0 = ang[0], a1 = ang[nview - 1], z0 = zsrc[0], z1 = zsrc[nview - 1];
    const float range = a1 - a0;
    if (fabsf(range) < 1.0e-6f) { *vs = 0; *ve = nview - 1; return; }
    const float db = range / fmaxf(1.0f, (float)(nview - 1));
    const float dzdb = (z1 - z0) / range;
    if (fabsf(db) < 1.0e-8f || fabsf(dzdb) < 1.0e-8f) { *vs = 0; *ve = nview - 1; return; }
    const float du = (float)g->du, dv = (float)g->dv, SOD = (float)g->sod, SDD = (float)g->sdd;
    const float gmax = du * (float)(g->Nu - 1) * 0.5f;
    const float half_scan = (XO_PI_F + 2.0f * gmax) * fmaxf(o->halfscan_coef, 1.0f);
    float span = 2.0f * XO_PI_F;
    if (o->view_mode == 1) span = half_scan;
    else if (o->view_mode == 2) span = 2.0f * XO_PI_F;
    else if (o->view_mode == 3) span = fmaxf(0.25f, o->view_turns) * 2.0f * XO_PI_F;
    else {
        const float ppt = fabsf(dzdb) * 2.0f * XO_PI_F;
        const float iso_h = fmaxf(dv * (float)g->Nv * SOD / SDD, dv);
        const float np = ppt / fmaxf(iso_h, 1.0e-6f);
        if (np >= 1.25f) span = half_scan;
        else if (np >= 0.45f) span = 2.0f * XO_PI_F;
        else if (np >= 0.25f) span = 3.0f * XO_PI_F;
        else span = 5.0f * XO_PI_F;
    }
    /* a window of V or more views is all views, and a centre beyond +-4V
     * gives the same clamped window as +-4V: both bounds keep the integer
     * arithmetic in range (the reference's values wherever it has them) */
    const float quot = span / fabsf(db);
    const float nwf = ceilf(o->window_quotient_up ? nextafterf(quot, INFINITY) : quot);
    const int nwin = (nwf >= (float)nview) ? nview : (nwf < 1.0f ? 1 : (int)nwf);
    const float bc = a0 + (pz - z0) / dzdb;
    const float vcf = roundf((bc - a0) / db);
    const int vc = (int)fminf(fmaxf(vcf, -4.0f * (float)nview), 4.0f * (float)nview);
    int s = vc - nwin / 2;
    if (s < 0) s = 0;
    int e = s + nwin - 1;
    if (e > nview - 1) e = nview - 1;
    s = e - nwin + 1;
    if (s < 0) s = 0;
    *vs = s; *ve = e;
}

/* helical_arc3d.cu:212-241 */
static float hw_conjugate(float beta, float gamma, float bc, float bs, float be, float db, float gmax)
{
    const float span = fabsf(be - bs);
    const float adb = fmaxf(fabsf(db), 1.0e-6f);
    if (span >= 2.0f * XO_PI_F - 2.0f * adb) {
        const float turns = fmaxf(1.0f, floorf((span + 2.0f * adb) / (2.0f * XO_PI_F)));
        return 0.5f * hw_center_turn(beta, bc, bs, be, db) / turns;
    }
    const float q = hw_window_quality(beta, bs, be, gamma, gmax);
    if (q <= 0.0f) return 0.0f;
    const float dir = (db >= 0.0f) ? 1.0f : -1.0f;
    float den = 0.0f;
    for (int k = -4; k <= 4; ++k) {
        const float turn = dir * 2.0f * XO_PI_F * (float)k;
        den += hw_window_quality(beta + turn, bs, be, gamma, gmax);
        den += hw_window_quality(beta + dir * (XO_PI_F + 2.0f * gamma) + turn, bs, be, -gamma, gmax);
    }
    return q / fmaxf(den, 1.0e-6f);
}

/* helical_arc3d.cu:243-303 */
static float hw_weight(float px, float py, float pz, float beta, float gamma, float src_z, float ray_xy, float bc,
                       float bs, float be, float db, float gmax, const float* ang, const float* zsrc, int nview,
                       const geo3_t* g, const hopt_t* o)
{
    if (o->weight_mode == 0) return hw_conjugate(beta, gamma, bc, bs, be, db, gmax);
    const float span = fabsf(be - bs);
    const float dir = (beta < bc) ? 1.0f : -1.0f;
    const float bcj = beta + dir * (XO_PI_F + 2.0f * gamma);
    float dq, cq;
    if (span < 2.0f * XO_PI_F - 2.0f * fabsf(db)) {
        dq = hw_window_quality(beta, bs, be, gamma, gmax);
        cq = hw_window_quality(bcj, bs, be, -gamma, gmax);
    } else {
        dq = hw_edge_taper(beta, bc, bs, be, db);
        cq = hw_edge_taper(bcj, bc, bs, be, db);
    }
    if (dq <= 0.0f) return 0.0f;
    if (cq <= 0.0f) return 1.0f;
    const float zc = hw_source_z_at(bcj, ang, zsrc, nview);
    const float SOD = (float)g->sod;
    const float sxc = -sinf(bcj) * SOD, syc = cosf(bcj) * SOD;
    const float rxc = px - sxc, ryc = py - syc;
    const float rxyc = sqrtf(rxc * rxc + ryc * ryc);
    const float ta = fabsf(pz - src_z) / fmaxf(ray_xy, 1.0e-6f);
    const float tac = fabsf(pz - zc) / fmaxf(rxyc, 1.0e-6f);
    const float k = fminf(fmaxf(o->tang_k, 0.0f), 32.0f);
    const float gg = powf(fmaxf(ta, 1.0e-6f), k);
    const float ggc = powf(fmaxf(tac, 1.0e-6f), k);
    const float w2 = dq / fmaxf(dq + cq, 1.0e-6f);
    const float den = dq * ggc + cq * gg;
    const float w3 = (dq * ggc) / fmaxf(den, 1.0e-6f);
    const float blend = hw_clamp_unit(o->tang_blend);
    return (1.0f - blend) * w2 + blend * w3;
}

/* Per-view float scalars of the weighted kernels (helical_arc3d.cu:1148-1160). */
typedef struct {
    float sod, sdd, du, shu, beta, sinv, cosv, sx, sy, szv;
} hwview_t;

static hwview_t hw_view(const geo3_t* g, const float* ang, const float* sp, int nview, int v)
{
    hwview_t w;
    const float sr = sp[nview + v], sa = sp[2 * nview + v];
    const float SOD = (float)g->sod, SDD = (float)g->sdd;
    w.sod = SOD + sr;
    w.sdd = SDD + sr;
    w.du = (float)g->du * SDD / w.sdd;
    w.shu = (float)g->shu * SDD / w.sdd - sa * (w.sdd - w.sod) / w.sdd;
    w.beta = ang[v] + sa;
    w.sinv = sinf(w.beta);
    w.cosv = cosf(w.beta);
    w.sx = -w.sinv * w.sod;
    w.sy = w.cosv * w.sod;
    w.szv = sp[v] + sp[3 * nview + v];
    return w;
}

/* helical_arc3d.cu:305-336 */
static int hw_measured(float px, float py, float pz, const hwview_t* w, float source_z_view, float shift_z,
                       const geo3_t* g)
{
    const float xb = w->cosv * px - w->sinv * py;
    const float yb = w->sinv * px + w->cosv * py;
    const float gamma = atan2f(yb, w->sod - xb);
    const float col = (gamma - w->shu) / w->du + (float)g->Nu * 0.5f - 0.5f;
    if (col < -0.5f || col > (float)g->Nu - 0.5f) return 0;
    const float src_z = source_z_view + shift_z;
    const float rx = px - w->sx, ry = py - w->sy;
    const float rxy = sqrtf(rx * rx + ry * ry);
    if (rxy <= 1.0e-6f) return 0;
    const float det_z = src_z + w->sdd * (pz - src_z) / rxy;
    const float row = (det_z - source_z_view - (float)g->shv) / (float)g->dv + (float)g->Nv * 0.5f - 0.5f;
    return row >= -0.5f && row <= (float)g->Nv - 0.5f;
}

/* View window of a z slice: [vs, ve], its end angles and centre angle. */
typedef struct {
    int vs, ve;
    float bs, be, bc;
} hzwin_t;

/* Redundancy weight of one (voxel, view) pair (helical_arc3d.cu:1148-1180);
 * *measured says whether the voxel centre projects onto the detector. */
static float hw_pair_weight(const geo3_t* g, const hopt_t* o, const float* ang, const float* sp, int nview,
                            const hzwin_t* zw, float db, float gmax, int ix, int iy, int iz, int v, int* measured)
{
    const float px = ((float)ix - (float)g->W / 2.0f + 0.5f) * (float)g->dx + (float)g->shx;
    const float py = ((float)g->H * 0.5f - (float)iy - 0.5f) * (float)g->dy + (float)g->shy;
    const float pz = ((float)iz - (float)g->D / 2.0f + 0.5f) * (float)g->dz + (float)g->shz;
    const hwview_t w = hw_view(g, ang, sp, nview, v);
    *measured = 0;
    const float rx = px - w.sx, ry = py - w.sy;
    const float rxy = sqrtf(rx * rx + ry * ry);
    if (rxy <= 1.0e-6f) return 0.0f;
    const float xb = w.cosv * px - w.sinv * py;
    const float yb = w.sinv * px + w.cosv * py;
    const float gamma = atan2f(yb, w.sod - xb);
    const float wt = hw_weight(px, py, pz, w.beta, gamma, w.szv, rxy, zw->bc, zw->bs, zw->be, db, gmax, ang, sp,
                               nview, g, o);
    if (wt != 0.0f) *measured = hw_measured(px, py, pz, &w, sp[v], sp[3 * nview + v], g);
    return wt;
}

/* Apply one helical operator.  fo = {view_mode, weight_mode, view_turns,
 * halfscan_coef, tang_k, tang_blend, window_quotient_up}; sp = source_pos
 * [4][nview]. */
int xo_helical3d(int op, const int* ni, const double* fv, const double* fg, const double* fo,
                 const double* in, double* out, const float* ang, const float* sp, int nbatch, int nview)
{
    geo3_t g;
    g.W = ni[0]; g.H = ni[1]; g.D = ni[2]; g.Nu = ni[3]; g.Nv = ni[4]; g.type = GEO_ARC;
    g.dx = fv[0]; g.dy = fv[1]; g.dz = fv[2]; g.shx = fv[3]; g.shy = fv[4]; g.shz = fv[5];
    g.du = fg[0]; g.dv = fg[1]; g.shu = fg[2]; g.shv = fg[3]; g.sod = fg[4]; g.sdd = fg[5];
    hopt_t o;
    o.view_mode = (int)fo[0]; o.weight_mode = (int)fo[1];
    o.view_turns = (float)fo[2]; o.halfscan_coef = (float)fo[3]; o.tang_k = (float)fo[4]; o.tang_blend = (float)fo[5];
    o.window_quotient_up = (int)fo[6];
    if (op < 0 || op > 5 || nview < 1) return 1;
    /* the helical column angles are evaluated exactly (their reference is
     * fast-math CUDA, not the float32 CPU arithmetic of arc_angle) */
    const int arc_exact_saved = g_arc_exact;
    g_arc_exact = 1;
    const long long nvox = (long long)g.W * g.H * g.D;
    const long long ncell = (long long)g.Nu * g.Nv;
    const int out_is_sino = (op == OP_A || op == OP_BT || op == OP_BWT);
    memset(out, 0, sizeof(double) * (size_t)nbatch * (size_t)(out_is_sino ? ncell * nview : nvox));
    const int weighted = (op == OP_BW || op == OP_BWT);

    /* weighted ops: per-slice windows and per-voxel scales */
    hzwin_t* zw = NULL;
    float* scale = NULL;
    const float db = (nview > 1) ? (ang[nview - 1] - ang[0]) / (float)(nview - 1) : 0.0f;
    const float gmax = (float)g.du * (float)(g.Nu - 1) * 0.5f;
    if (weighted) {
        zw = malloc(sizeof(hzwin_t) * g.D);
        scale = malloc(sizeof(float) * (size_t)nvox);
        for (int iz = 0; iz < g.D; ++iz) {
            const float pz = ((float)iz - (float)g.D / 2.0f + 0.5f) * (float)g.dz + (float)g.shz;
            hw_view_window(pz, ang, sp, &g, &o, nview, &zw[iz].vs, &zw[iz].ve);
            zw[iz].bs = ang[zw[iz].vs];
            zw[iz].be = ang[zw[iz].ve];
            zw[iz].bc = hw_center_beta(pz, ang, sp, zw[iz].vs, zw[iz].ve, nview);
        }
        for (int iz = 0; iz < g.D; ++iz)
            for (int iy = 0; iy < g.H; ++iy)
                for (int ix = 0; ix < g.W; ++ix) {
                    float valid = 0.0f;
                    for (int v = zw[iz].vs; v <= zw[iz].ve; ++v) {
                        int meas;
                        const float wt = hw_pair_weight(&g, &o, ang, sp, nview, &zw[iz], db, gmax, ix, iy, iz, v, &meas);
                        if (wt != 0.0f && meas) valid += wt;
                    }
                    const float ideal = (fabsf(db) > 1.0e-8f) ? (XO_PI_F / fabsf(db)) : valid;
                    float s = ideal / fmaxf(valid, 1.0e-6f);
                    s = fminf(32.0f, fmaxf(0.03125f, s));
                    scale[((long long)iz * g.H + iy) * g.W + ix] = s;
                }
    }
    const double cwW = (double)((float)g.sod * (float)g.du);   /* helical_arc3d.cu:1144 */

    const int nline_max = g.W > g.H ? g.W : g.H;
    double* D = malloc(sizeof(double) * (g.Nu + 1));
    double* M = malloc(sizeof(double) * g.Nu);
    double* zd = malloc(sizeof(double) * (g.Nv + 1));
    double* X = malloc(sizeof(double) * (nline_max + 1));
    double* Zv = malloc(sizeof(double) * (g.D + 1));
    double* Zc = malloc(sizeof(double) * (g.Nv + 1));
    const int nxo = nline_max + g.Nu + 2, nzo = g.D + g.Nv + 2;
    int* xa = malloc(sizeof(int) * nxo); int* xb = malloc(sizeof(int) * nxo);
    double* xl = malloc(sizeof(double) * nxo);
    int* za = malloc(sizeof(int) * nzo); int* zb = malloc(sizeof(int) * nzo);
    double* zl = malloc(sizeof(double) * nzo);
    const double z0 = -0.5 * g.D * g.dz + g.shz;

    for (int view = 0; view < nview; ++view) {
        hview_t hv;
        helical_view(&g, ang, sp, nview, view, &hv);
        const geo3_t* gv = &hv.g;
        const view_t* v = &hv.v;
        view_columns3d(gv, v, D, M, zd);
        for (int r = 0; r <= g.Nv; ++r) zd[r] = hv.zrow0 + r * g.dv;
        const double dperp = v->use_x ? g.dy : g.dx;
        const int nlines = v->use_x ? g.H : g.W;
        for (int line = 0; line < nlines; ++line) {
            double Mv, perp;
            const int npix = line_pixels3d(gv, v, line, X, &Mv, &perp);
            for (int i = 0; i <= g.D; ++i) Zv[i] = Mv * (z0 - hv.zsrc + i * g.dz);
            const int nx = overlaps(X, npix, D, g.Nu, xa, xb, xl);
            for (int e = 0; e < nx; ++e) {
                const int p = xa[e], k = xb[e];
                const int ix = v->use_x ? p : line;
                const int iy = v->use_x ? line : g.H - 1 - p;
                const int col = v->keep ? k : g.Nu - 1 - k;
                for (int r = 0; r <= g.Nv; ++r) Zc[r] = M[k] * zd[r];
                const int nz = overlaps(Zv, g.D, Zc, g.Nv, za, zb, zl);
                const double pixz = (X[p + 1] - X[p]) * Mv * g.dz;
                double fbpw = 0.0;
                if (weighted) {
                    double px, py;
                    voxel_xy(&g, ix, iy, &px, &py);
                    const double ex = v->sx - px, ey = v->sy - py;
                    fbpw = cwW / (pixz * (ex * ex + ey * ey));
                }
                for (int q = 0; q < nz; ++q) {
                    const int iz = za[q], r = zb[q];
                    const double coef = xl[e] * zl[q];
                    double s;
                    if (op == OP_A || op == OP_AT) {
                        const double dD = D[k + 1] - D[k];
                        const double dZ = Zc[r + 1] - Zc[r];
                        const double a = 0.5 * (D[k + 1] + D[k]) - v->spar;
                        const double b = 0.5 * (Zc[r + 1] + Zc[r]) + hv.zsrc;
                        const double cosw = fabs(v->sperp) / sqrt(a * a + b * b + v->sperp * v->sperp);
                        s = dperp / (dD * dZ * cosw);
                    } else if (!weighted) {
                        s = hv.cwB / pixz;
                    } else {
                        if (view < zw[iz].vs || view > zw[iz].ve) continue;
                        int meas;
                        const float wt = hw_pair_weight(&g, &o, ang, sp, nview, &zw[iz], db, gmax, ix, iy, iz, view,
                                                        &meas);
                        if (wt == 0.0f) continue;
                        s = fbpw * (double)wt * (double)scale[((long long)iz * g.H + iy) * g.W + ix];
                    }
                    for (int bt = 0; bt < nbatch; ++bt) {
                        const long long vi = ((long long)(bt * g.D + iz) * g.H + iy) * g.W + ix;
                        const long long ci = (((long long)bt * nview + view) * g.Nv + r) * g.Nu + col;
                        switch (op) {
                        case OP_A:   out[ci] += coef * s * in[vi]; break;
                        case OP_AT:
                        case OP_B:
                        case OP_BW:  out[vi] += coef * s * in[ci]; break;
                        default:     out[ci] += coef * s * in[vi]; break;
                        }
                    }
                }
            }
        }
    }
    free(D); free(M); free(zd); free(X); free(Zv); free(Zc);
    free(xa); free(xb); free(xl); free(za); free(zb); free(zl);
    free(zw); free(scale);
    g_arc_exact = arc_exact_saved;
    return 0;
}
