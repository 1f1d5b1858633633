// Test infrastructure only: a C-ABI shim over the reference's own CPU
// implementation (XRecon src/cpu/*.cpp), compiled from the reference sources
// in place by oracle/build_oracle.py into oracle/_ref/.  Nothing in the
// product links this; tests and the bench's CPU reference arm load it with
// ctypes.
//
// Each entry point forwards to the reference function named beside it and
// builds the reference's Volume/Geometry structs (include/types.h:35-119)
// from plain scalars, exactly as the reference binding does after unpacking
// the options tensor (src/api/torch_binding.cpp:62-124).
#include <vector>

#include "types.h"
#include "functions.h"

namespace {

xrecon::Volume2d make_vol2d(int W, int H, float dx, float dy, float shx, float shy) {
    return xrecon::Volume2d(W, H, dx, dy, shx, shy);
}

xrecon::Geometry2d make_geo2d(int type, int Nu, float du, float shu, float sod, float sdd) {
    return xrecon::Geometry2d(static_cast<xrecon::GeometryType>(type), Nu, du, shu, sod, sdd);
}

xrecon::Volume3d make_vol3d(const int* n, const float* f) {
    // n = {W, H, D}; f = {dx, dy, dz, shx, shy, shz}
    return xrecon::Volume3d(n[0], n[1], n[2], f[0], f[1], f[2], f[3], f[4], f[5]);
}

xrecon::Geometry3d make_geo3d(int type, const int* n, const float* f) {
    // n = {Nu, Nv}; f = {du, dv, shu, shv, SOD, SDD}
    return xrecon::Geometry3d(static_cast<xrecon::GeometryType>(type), n[0], n[1],
                              f[0], f[1], f[2], f[3], f[4], f[5]);
}

}  // namespace

extern "C" {

// op: 0 projection (forward2d_cpu), 1 projection transpose (forward2d_t_cpu),
//     2 backprojection (backward2d_cpu), 3 backprojection transpose
//     (backward2d_t_cpu), 4 weighted backprojection (weighted_backward2d_cpu),
//     5 weighted backprojection transpose (weighted_backward2d_t_cpu).
// Declarations: include/functions.h:72-169 of the reference.
int xr_ref_dd2d(int op, float* image, float* proj, float* ang,
                int W, int H, float dx, float dy, float shx, float shy,
                int type, int Nu, float du, float shu, float sod, float sdd,
                int nbatch, int nview)
{
    const xrecon::Volume2d vol = make_vol2d(W, H, dx, dy, shx, shy);
    const xrecon::Geometry2d geo = make_geo2d(type, Nu, du, shu, sod, sdd);
    switch (op) {
    case 0: xrecon::forward2d_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 1: xrecon::forward2d_t_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 2: xrecon::backward2d_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 3: xrecon::backward2d_t_cpu(proj, image, ang, vol, geo, nbatch, nview); return 0;
    case 4: xrecon::weighted_backward2d_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 5: xrecon::weighted_backward2d_t_cpu(proj, image, ang, vol, geo, nbatch, nview); return 0;
    default: return 1;
    }
}

// Same op numbering, 3D functions of include/functions.h:249-254.
// ni = {W, H, D, Nu, Nv}; fv = {dx, dy, dz, shx, shy, shz};
// fg = {du, dv, shu, shv, SOD, SDD} in the packed (options-tensor) units.
int xr_ref_dd3d(int op, float* image, float* proj, float* ang,
                const int* ni, const float* fv, const float* fg, int type,
                int nbatch, int nview)
{
    const xrecon::Volume3d vol = make_vol3d(ni, fv);
    const xrecon::Geometry3d geo = make_geo3d(type, ni + 3, fg);
    switch (op) {
    case 0: xrecon::forward3d_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 1: xrecon::forward3d_t_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 2: xrecon::backward3d_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 3: xrecon::backward3d_t_cpu(proj, image, ang, vol, geo, nbatch, nview); return 0;
    case 4: xrecon::weighted_backward3d_cpu(image, proj, ang, vol, geo, nbatch, nview); return 0;
    case 5: xrecon::weighted_backward3d_t_cpu(proj, image, ang, vol, geo, nbatch, nview); return 0;
    default: return 1;
    }
}

// System matrix of the projection (system_matrix2d_cpu /
// system_matrix3d_cpu, include/functions.h:92-118): fills at most `cap`
// triplets and returns their total count (call again with a larger buffer
// when the count exceeds cap), or -1 on an unknown geometry.
long long xr_ref_sysmat2d(float* ang, int W, int H, float dx, float dy, float shx, float shy, int type, int Nu,
                          float du, float shu, float sod, float sdd, int nview, long long* rows, long long* cols,
                          float* vals, long long cap)
{
    if (type < 0 || type > 2) return -1;
    std::vector<int64_t> r, c;
    std::vector<float> v;
    xrecon::system_matrix2d_cpu(r, c, v, ang, make_vol2d(W, H, dx, dy, shx, shy),
                                make_geo2d(type, Nu, du, shu, sod, sdd), nview);
    const long long n = (long long)v.size();
    for (long long i = 0; i < n && i < cap; ++i) { rows[i] = r[i]; cols[i] = c[i]; vals[i] = v[i]; }
    return n;
}

long long xr_ref_sysmat3d(float* ang, const int* ni, const float* fv, const float* fg, int type, int nview,
                          long long* rows, long long* cols, float* vals, long long cap)
{
    if (type < 0 || type > 2) return -1;
    std::vector<int64_t> r, c;
    std::vector<float> v;
    xrecon::system_matrix3d_cpu(r, c, v, ang, make_vol3d(ni, fv), make_geo3d(type, ni + 3, fg), nview);
    const long long n = (long long)v.size();
    for (long long i = 0; i < n && i < cap; ++i) { rows[i] = r[i]; cols[i] = c[i]; vals[i] = v[i]; }
    return n;
}

}  // extern "C"
