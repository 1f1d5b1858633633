// Test infrastructure only: a C entry point over the reference's own helical
// CUDA launchers (XRecon src/kernels/helical_arc3d.cu:1763-1983), compiled
// together with that file into oracle/_ref/ by oracle/build_oracle.py.  The
// fixture generator tests/golden/make_golden_helical.py calls it on a GPU to
// record the reference's helical outputs; nothing in the product links it.
//
// The Volume3d / Geometry3d values are built from the 24 packed options as
// the reference binding builds them (src/api/torch_binding.cpp:82-124), and
// source_pos is split into its four rows as launch_helical_arc3d does
// (torch_binding.cpp:128-138).
#include <cuda_runtime.h>

#include "types.h"

using HelicalFn = void (*)(float*, float*, float*, float*, float*, float*, float*, int, xrecon::Volume3d,
                           xrecon::Geometry3d, int);

void helical_arc_forward_cuda(float*, float*, float*, float*, float*, float*, float*, int, xrecon::Volume3d,
                              xrecon::Geometry3d, int);
void helical_arc_forward_t_cuda(float*, float*, float*, float*, float*, float*, float*, int, xrecon::Volume3d,
                                xrecon::Geometry3d, int);
void helical_arc_backward_cuda(float*, float*, float*, float*, float*, float*, float*, int, xrecon::Volume3d,
                               xrecon::Geometry3d, int);
void helical_arc_backward_t_cuda(float*, float*, float*, float*, float*, float*, float*, int, xrecon::Volume3d,
                                 xrecon::Geometry3d, int);
void helical_arc_weighted_backward_cuda(float*, float*, float*, float*, float*, float*, float*, int,
                                        xrecon::Volume3d, xrecon::Geometry3d, int);
void helical_arc_weighted_backward_t_cuda(float*, float*, float*, float*, float*, float*, float*, int,
                                          xrecon::Volume3d, xrecon::Geometry3d, int);

// op: 0 A, 1 A^T, 2 B, 3 B^T, 4 Bw, 5 Bw^T (the reference's six bindings).
// opts: host float[24]; image, proj, angles, source_pos: device float32.
// The caller zero-fills the output of A^T, B, Bw and Bw^T (the reference's
// kernels accumulate into it).  Returns the CUDA error code after a
// device synchronisation.
extern "C" int xr_ref_helical(int op, const float* opts, float* image, float* proj, float* angles,
                              float* source_pos, int nbatch, int nview) {
    static const HelicalFn fns[6] = {helical_arc_forward_cuda, helical_arc_forward_t_cuda,
                                     helical_arc_backward_cuda, helical_arc_backward_t_cuda,
                                     helical_arc_weighted_backward_cuda, helical_arc_weighted_backward_t_cuda};
    if (op < 0 || op > 5 || nview < 1 || nbatch < 1) return -1;
    const xrecon::Volume3d vol((int)opts[0], (int)opts[1], (int)opts[2], opts[5], opts[6], opts[7], opts[12],
                               opts[13], opts[14]);
    const xrecon::Geometry3d geo(static_cast<xrecon::GeometryType>((int)opts[17]), (int)opts[3], (int)opts[4],
                                 opts[8], opts[9], opts[15], opts[16], opts[10], opts[11], (int)opts[18],
                                 (int)opts[19], opts[20], opts[21], opts[22], opts[23]);
    fns[op](image, proj, angles, source_pos, source_pos + nview, source_pos + 2 * nview, source_pos + 3 * nview,
            nbatch, vol, geo, nview);
    const cudaError_t e = cudaDeviceSynchronize();
    return e != cudaSuccess ? (int)e : (int)cudaGetLastError();
}
