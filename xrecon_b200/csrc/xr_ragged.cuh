// Ragged batch of 2D reconstructions (projection then FBP) in one persistent
// cooperative launch.
//
// Every instance has its own geometry, image size, view count and detector.
// The kernel runs four phases over a list of tiles that spans all instances;
// each block takes tiles from a per-phase atomic counter, so instances of
// very different cost share the GPU without idle SMs.  Phases are separated
// by a grid barrier whose waits are bounded (a timeout sets the device error
// word and ends the kernel):
//   0  per-view DD tables of every instance (FP64) and the flipped transpose
//      of every image (lines of y-axis views);
//   1  projection A, cell-owned: a tile is CW columns of one view, the
//      256 / CW threads of a column split its lines and reduce in shared
//      memory;
//   2  FBP pre-filter of every sinogram row: cosine weight x correlation with
//      the instance's filter taps (the same arithmetic as fbp_filter_kernel);
//   3  weighted backprojection Bw of the filtered rows times the FBP scale,
//      pixel-owned: a tile is 256 / VS pixels, the VS threads of a pixel
//      split its views and reduce in shared memory.
// CW and VS are launch parameters chosen by the autotuner of the Python
// wrapper.  No atomics touch data: the counters only hand out tiles.
#pragma once

#include "xr_kernels.cuh"
#include "xr_tma.cuh"

namespace xr {

constexpr unsigned XR_DEVERR_BARRIER_TIMEOUT = 2u;
// polls of ~128 ns: about half a second by default (xr_set_wait_limits)
constexpr long long XR_BARRIER_LIMIT_DEFAULT = 1ll << 22;
__device__ long long g_barrier_limit = XR_BARRIER_LIMIT_DEFAULT;

// One instance, device side (pointers already resolved).
struct RaggedDev {
    Geom g;
    ViewTables vt;
    int nview;
    float cw;       // backprojection column width
    float scale;    // FBP scale
    const float* img;
    float* imgT;
    float* sino;
    float* filt_out;
    float* recon;
    const float* ang;
    const float* filt;
    const float* cosw;
    // first tile of this instance in each tile list: [0] tables and
    // transposes, [1] filter rows, [2 + i] projection with CW = 32 << i,
    // [6 + i] backprojection with VS = 1 << i
    int t0[10];
};

// Bounded grid barrier over nblocks co-resident blocks; bar[0] counts
// arrivals, bar[1] is the generation.  False when a wait gave up.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned nblocks) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u) + 1u;
        const long long limit = *(volatile long long*)&g_barrier_limit;
        // test hook: one block more than the grid is expected, nobody releases
        if (*(volatile unsigned*)&g_test_hooks & XR_HOOK_BARRIER_EXTRA) ++nblocks;
        int ok = 1;
        if (arrived == nblocks) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long i = 0;
            while (*vgen == gen) {
                if (++i > limit) {
                    atomicOr(&g_device_error, XR_DEVERR_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// Instance owning global tile t of tile list p (t0[p] ascending).
__device__ __forceinline__ int find_instance(const RaggedDev* __restrict__ inst, int ninst, int p, int t) {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (inst[mid].t0[p] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int next_tile(int* ctr) {
    __shared__ int t_s;
    __syncthreads();
    if (threadIdx.x == 0) t_s = atomicAdd(ctr, 1);
    __syncthreads();
    return t_s;
}

__global__ void __launch_bounds__(256, 3)
ragged2d_fbp_kernel(const RaggedDev* __restrict__ inst, const int ninst, const int4 totals, const int4 lists,
                    const int project, const int CW, const int VS, unsigned* bar, int* ctr) {
    extern __shared__ float sm[];
    const int tid = threadIdx.x;
    const unsigned nb = gridDim.x;

    // phase 0: view tables and transposes
    for (int t = next_tile(&ctr[0]); t < totals.x; t = next_tile(&ctr[0])) {
        const RaggedDev& I = inst[find_instance(inst, ninst, lists.x, t)];
        const int lt = t - I.t0[lists.x];
        const Geom& g = I.g;
        if (lt < I.nview) {
            for (int k = tid; k <= g.Nu; k += blockDim.x) setup_view_entry(g, 0, I.ang[lt], lt, k, I.vt, g.type == GEO_ARC);
        } else {
            const int base = (lt - I.nview) * 1024;
            for (int e = tid; e < 1024; e += blockDim.x) {
                const int idx = base + e;
                if (idx < g.H * g.W) {
                    const int y = idx / g.W, x = idx - y * g.W;
                    I.imgT[(size_t)x * g.H + (g.H - 1 - y)] = I.img[idx];
                }
            }
        }
    }
    if (!grid_barrier(bar, nb)) return;

    // phase 1: projection
    if (project) {
        const int LS = blockDim.x / CW;
        for (int t = next_tile(&ctr[1]); t < totals.y; t = next_tile(&ctr[1])) {
            const RaggedDev& I = inst[find_instance(inst, ninst, lists.y, t)];
            const Geom& g = I.g;
            const int nbk = (g.Nu + CW - 1) / CW;
            const int lt = t - I.t0[lists.y];
            const int v = lt / nbk, kb = lt - v * nbk;
            const int c = tid % CW, s = tid / CW;
            const int k = kb * CW + c;
            const ViewHdr h = I.vt.hdr[v];
            float acc = 0.0f;
            if (k < g.Nu) acc = cell2d_sum<float, OP_A>(g, I.vt, h, I.img, I.imgT, v, k, 0.0f, s, LS);
            sm[tid] = acc;
            __syncthreads();
            if (s == 0 && k < g.Nu) {
                float sum = 0.0f;
                for (int j = 0; j < LS; ++j) sum += sm[j * CW + c];
                if (LS > 1) sum *= I.vt.colE[(size_t)v * g.Nu + k];  // LS == 1: applied by cell2d_sum
                const int col = h.keep ? k : g.Nu - 1 - k;
                I.sino[(size_t)v * g.Nu + col] = sum;
            }
        }
    }
    if (!grid_barrier(bar, nb)) return;

    // phase 2: cosine weight x filter correlation, one sinogram row per tile
    for (int t = next_tile(&ctr[2]); t < totals.z; t = next_tile(&ctr[2])) {
        const RaggedDev& I = inst[find_instance(inst, ninst, lists.z, t)];
        const int Nu = I.g.Nu;
        const int v = t - I.t0[lists.z];
        float* x = sm;             // Nu
        float* f = sm + Nu;        // 2 Nu - 1
        for (int j = tid; j < Nu; j += blockDim.x) x[j] = I.sino[(size_t)v * Nu + j] * I.cosw[j];
        for (int j = tid; j < 2 * Nu - 1; j += blockDim.x) f[j] = I.filt[j];
        __syncthreads();
        for (int i = tid; i < Nu; i += blockDim.x) {
            // out[i] = sum_j x[j] f[j - i + Nu - 1]
            const float* fi = f + (Nu - 1 - i);
            float a0 = 0.0f, a1 = 0.0f;
            int j = 0;
            for (; j + 1 < Nu; j += 2) {
                a0 = fmaf(x[j], fi[j], a0);
                a1 = fmaf(x[j + 1], fi[j + 1], a1);
            }
            if (j < Nu) a0 = fmaf(x[j], fi[j], a0);
            I.filt_out[(size_t)v * Nu + i] = a0 + a1;
        }
    }
    if (!grid_barrier(bar, nb)) return;

    // phase 3: weighted backprojection x FBP scale
    {
        const int PX = blockDim.x / VS;
        for (int t = next_tile(&ctr[3]); t < totals.w; t = next_tile(&ctr[3])) {
            const RaggedDev& I = inst[find_instance(inst, ninst, lists.w, t)];
            const Geom& g = I.g;
            const int p = tid % PX, s = tid / PX;
            const int idx = (t - I.t0[lists.w]) * PX + p;
            float acc = 0.0f;
            if (idx < g.H * g.W) {
                const int iy = idx / g.W, ix = idx - iy * g.W;
                acc = pix2d_sum<float, OP_BW>(g, I.vt, I.filt_out, ix, iy, I.cw, s, I.nview, VS);
            }
            sm[tid] = acc;
            __syncthreads();
            if (s == 0 && idx < g.H * g.W) {
                float sum = 0.0f;
                for (int j = 0; j < VS; ++j) sum += sm[j * PX + p];
                I.recon[idx] = sum * I.scale;
            }
        }
    }
    // leave the tile counters at zero for the next launch
    if (!grid_barrier(bar, nb)) return;
    if (blockIdx.x == 0 && tid < 4) ctr[tid] = 0;
}

}  // namespace xr
