// FBP filter by FFT.
//
// The filter is the correlation out[i] = sum_j x[j] filt[j - i + Nu - 1]
// (conv with padding Nu - 1: projector.py:201, projector3d.py:190).  With
// M a power of two >= 2 Nu - 1 every lag j - i in [-(Nu - 1), Nu - 1] has
// its own residue mod M, so the correlation is the circular convolution of x
// (zero-padded to M) with g[(Nu - 1 - t) mod M] = filt[t]:
//     out = IFFT(FFT(x) * FFT(g)).
// Two rows share one complex transform (z = x1 + i x2): FFT(g) is the
// transform of a real sequence, so the real and imaginary parts of
// IFFT(FFT(z) FFT(g)) are the two filtered rows.
//
// One CTA owns four rows (two transforms) at a time in shared memory.  The
// forward transform is decimation in frequency (natural order in,
// bit-reversed out), the inverse decimation in time (bit-reversed in, natural
// out), so no pass permutes: the spectrum of g is kept in the same
// bit-reversed order.  The
// inverse is a forward transform of the conjugate, IFFT(Y) = conj(FFT(conj
// Y)) / M.  Stages are fused in pairs (radix 4); an odd power of two adds one
// radix-2 stage.  Rows are FP32 with FP32 twiddles (rounded from FP64); each
// CTA transforms g once in FP64.  Round-off is of order eps log2(M) of the
// row's norm, where the direct sum's is eps sqrt(Nu) of its terms.
#pragma once

#include "xr_kernels.cuh"

namespace xr {

constexpr int XR_FFT_THREADS = 256;
constexpr int XR_FFT_MAX_LOG = 12;  // M <= 4096, so Nu <= 2048

__host__ __device__ inline int fft_log2_for(int Nu) {
    int m = 1;
    while ((1 << m) < 2 * Nu - 1) ++m;
    return m;
}

// Radix-4 stage pairs of a length-2^m transform work on groups of 4h with
// h = h0, 4 h0, ..., M / 4 (h0 = 2 for odd m, else 1); both directions use
// the same h.  Their FP32 twiddles {W_2h^j, W_4h^j}, j < h, are stored per
// stage, contiguous in j, at fft_tw_offset(h): a warp's lanes then read
// neighbouring entries instead of entries M / 2h apart, which fall on one
// shared-memory bank.
__host__ __device__ inline int fft_h0(int m) { return (m & 1) ? 2 : 1; }
__host__ __device__ inline int fft_tw_offset(int h, int m) { return (h - fft_h0(m)) / 3; }
__host__ __device__ inline int fft_tw_count(int m) { return ((1 << m) - fft_h0(m)) / 3; }

// Shared memory: the data (double2 while g is transformed, then two float2
// row buffers), the FP64 twiddles of that transform (then the spectrum of
// g, the same size), the per-stage FP32 twiddles.
__host__ __device__ inline size_t fft_filter_smem(int m) {
    const size_t M = (size_t)1 << m;
    return M * sizeof(double2) + (M / 2) * sizeof(double2) + (size_t)fft_tw_count(m) * sizeof(float4);
}

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 c_mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)
__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 c_mul_mi(double2 a) { return make_double2(a.y, -a.x); }

// Forward DFT of a[0..M), decimation in frequency: natural order in,
// bit-reversed order out.  tw[k] = exp(-2 pi i k / M), k < M / 2.  Ends with
// a barrier.
template <typename C>
__device__ void fft_dif(C* a, const C* __restrict__ tw, const int m) {
    const int M = 1 << m;
    for (int h = M / 4; h >= 1; h /= 4) {
        // stages of half-size 2h then h, on groups of 4h elements
        const int s1 = M / (2 * h), s2 = M / (4 * h);
        for (int i = threadIdx.x; i < M / 4; i += blockDim.x) {
            const int j = i & (h - 1), base = (i - j) * 4 + j;
            const C x0 = a[base], x1 = a[base + h], x2 = a[base + 2 * h], x3 = a[base + 3 * h];
            const C w1 = tw[j * s1], w2 = tw[j * s2];
            const C y0 = c_add(x0, x2), y2 = c_mul(c_sub(x0, x2), w2);
            const C y1 = c_add(x1, x3), y3 = c_mul(c_mul_mi(c_sub(x1, x3)), w2);
            a[base] = c_add(y0, y1);
            a[base + h] = c_mul(c_sub(y0, y1), w1);
            a[base + 2 * h] = c_add(y2, y3);
            a[base + 3 * h] = c_mul(c_sub(y2, y3), w1);
        }
        __syncthreads();
    }
    if (m & 1) {  // last stage of half-size 1 (twiddle 1)
        for (int i = threadIdx.x; i < M / 2; i += blockDim.x) {
            const C x0 = a[2 * i], x1 = a[2 * i + 1];
            a[2 * i] = c_add(x0, x1);
            a[2 * i + 1] = c_sub(x0, x1);
        }
        __syncthreads();
    }
}

// Forward DFT, decimation in time: bit-reversed order in, natural order out.
// Ends with a barrier.
template <typename C>
__device__ void fft_dit(C* a, const C* __restrict__ tw, const int m) {
    const int M = 1 << m;
    int h = 1;
    if (m & 1) {  // first stage of half-size 1 (twiddle 1)
        for (int i = threadIdx.x; i < M / 2; i += blockDim.x) {
            const C x0 = a[2 * i], x1 = a[2 * i + 1];
            a[2 * i] = c_add(x0, x1);
            a[2 * i + 1] = c_sub(x0, x1);
        }
        __syncthreads();
        h = 2;
    }
    for (; h < M; h *= 4) {
        // stages of half-size h then 2h, on groups of 4h elements
        const int s1 = M / (2 * h), s2 = M / (4 * h);
        for (int i = threadIdx.x; i < M / 4; i += blockDim.x) {
            const int j = i & (h - 1), base = (i - j) * 4 + j;
            const C x0 = a[base], x1 = a[base + h], x2 = a[base + 2 * h], x3 = a[base + 3 * h];
            const C w1 = tw[j * s1], w2 = tw[j * s2];
            const C t1 = c_mul(x1, w1), t3 = c_mul(x3, w1);
            const C y0 = c_add(x0, t1), y1 = c_sub(x0, t1);
            const C y2 = c_add(x2, t3), y3 = c_sub(x2, t3);
            const C u2 = c_mul(y2, w2), u3 = c_mul_mi(c_mul(y3, w2));
            a[base] = c_add(y0, u2);
            a[base + 2 * h] = c_sub(y0, u2);
            a[base + h] = c_add(y1, u3);
            a[base + 3 * h] = c_sub(y1, u3);
        }
        __syncthreads();
    }
}

// fft_dif / fft_dit on NB consecutive FP32 arrays of length M at once (one
// barrier per stage pair for all of them), with the per-stage twiddles.
template <int NB>
__device__ void fft_dif_rows(float2* a, const float4* __restrict__ tws, const int m) {
    const int M = 1 << m;
    for (int h = M / 4; h >= 1; h /= 4) {
        const float4* __restrict__ th = tws + fft_tw_offset(h, m);
        for (int i = threadIdx.x; i < NB * (M / 4); i += blockDim.x) {
            const int f = i >> (m - 2), ii = i & (M / 4 - 1);
            const int j = ii & (h - 1), base = f * M + (ii - j) * 4 + j;
            const float2 x0 = a[base], x1 = a[base + h], x2 = a[base + 2 * h], x3 = a[base + 3 * h];
            const float4 w = th[j];
            const float2 w1 = make_float2(w.x, w.y), w2 = make_float2(w.z, w.w);
            const float2 y0 = c_add(x0, x2), y2 = c_mul(c_sub(x0, x2), w2);
            const float2 y1 = c_add(x1, x3), y3 = c_mul(c_mul_mi(c_sub(x1, x3)), w2);
            a[base] = c_add(y0, y1);
            a[base + h] = c_mul(c_sub(y0, y1), w1);
            a[base + 2 * h] = c_add(y2, y3);
            a[base + 3 * h] = c_mul(c_sub(y2, y3), w1);
        }
        __syncthreads();
    }
    if (m & 1) {
        for (int i = threadIdx.x; i < NB * (M / 2); i += blockDim.x) {
            const float2 x0 = a[2 * i], x1 = a[2 * i + 1];
            a[2 * i] = c_add(x0, x1);
            a[2 * i + 1] = c_sub(x0, x1);
        }
        __syncthreads();
    }
}

template <int NB>
__device__ void fft_dit_rows(float2* a, const float4* __restrict__ tws, const int m) {
    const int M = 1 << m;
    int h = 1;
    if (m & 1) {
        for (int i = threadIdx.x; i < NB * (M / 2); i += blockDim.x) {
            const float2 x0 = a[2 * i], x1 = a[2 * i + 1];
            a[2 * i] = c_add(x0, x1);
            a[2 * i + 1] = c_sub(x0, x1);
        }
        __syncthreads();
        h = 2;
    }
    for (; h < M; h *= 4) {
        const float4* __restrict__ th = tws + fft_tw_offset(h, m);
        for (int i = threadIdx.x; i < NB * (M / 4); i += blockDim.x) {
            const int f = i >> (m - 2), ii = i & (M / 4 - 1);
            const int j = ii & (h - 1), base = f * M + (ii - j) * 4 + j;
            const float2 x0 = a[base], x1 = a[base + h], x2 = a[base + 2 * h], x3 = a[base + 3 * h];
            const float4 w = th[j];
            const float2 w1 = make_float2(w.x, w.y), w2 = make_float2(w.z, w.w);
            const float2 t1 = c_mul(x1, w1), t3 = c_mul(x3, w1);
            const float2 y0 = c_add(x0, t1), y1 = c_sub(x0, t1);
            const float2 y2 = c_add(x2, t3), y3 = c_sub(x2, t3);
            const float2 u2 = c_mul(y2, w2), u3 = c_mul_mi(c_mul(y3, w2));
            a[base] = c_add(y0, u2);
            a[base + 2 * h] = c_sub(y0, u2);
            a[base + h] = c_add(y1, u3);
            a[base + 3 * h] = c_sub(y1, u3);
        }
        __syncthreads();
    }
}

// One CTA per four rows at a time (grid-stride): two complex transforms
// side by side.  Rows is a row source as for fbp_filter_kernel (weights
// applied on load).
template <typename Rows>
__global__ void __launch_bounds__(XR_FFT_THREADS)
fft_filter_kernel(const Rows src, float* __restrict__ out, const int nrows, const int Nu,
                  const float* __restrict__ filt, const int m) {
    extern __shared__ __align__(16) unsigned char fsm[];
    const int M = 1 << m;
    double2* d64 = reinterpret_cast<double2*>(fsm);              // [M], FP64 setup
    float2* rows = reinterpret_cast<float2*>(fsm);                // [2][M], aliases d64 afterwards
    double2* tw64 = reinterpret_cast<double2*>(fsm + (size_t)M * sizeof(double2));  // [M / 2], setup
    float2* spec = reinterpret_cast<float2*>(tw64);               // [M], aliases tw64 afterwards
    float4* tws = reinterpret_cast<float4*>(fsm + (size_t)M * sizeof(double2) + (size_t)(M / 2) * sizeof(double2));
    const int tid = threadIdx.x, nt = blockDim.x;

    // twiddles, and g in natural order
    for (int k = tid; k < M / 2; k += nt) {
        double s, c;
        sincospi(-2.0 * (double)k / (double)M, &s, &c);
        tw64[k] = make_double2(c, s);
    }
    for (int h = fft_h0(m); h <= M / 4; h *= 4) {
        for (int j = tid; j < h; j += nt) {
            double s1, c1, s2, c2;
            sincospi(-(double)j / (double)h, &s1, &c1);          // W_2h^j
            sincospi(-(double)j / (double)(2 * h), &s2, &c2);    // W_4h^j
            tws[fft_tw_offset(h, m) + j] = make_float4((float)c1, (float)s1, (float)c2, (float)s2);
        }
    }
    for (int n = tid; n < M; n += nt) {
        const int t = (n <= Nu - 1) ? Nu - 1 - n : M + Nu - 1 - n;  // (Nu - 1 - n) mod M
        d64[n] = make_double2(t <= 2 * Nu - 2 ? (double)filt[t] : 0.0, 0.0);
    }
    __syncthreads();
    fft_dif(d64, tw64, m);
    // spectrum of g, bit-reversed, with the inverse's 1 / M, over tw64 (no
    // longer read: fft_dif ended with a barrier); the row buffers take d64's
    // place only after the next barrier
    const double inv_m = 1.0 / (double)M;
    for (int k = tid; k < M; k += nt) spec[k] = make_float2((float)(d64[k].x * inv_m), (float)(d64[k].y * inv_m));
    __syncthreads();

    const int nquad = (nrows + 3) / 4;
    for (int q = blockIdx.x; q < nquad; q += gridDim.x) {
        const int r0 = 4 * q;
        for (int n = tid; n < M; n += nt) {
            float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (n < Nu) {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (r0 + e < nrows) x[e] = src(r0 + e, n);
            }
            rows[n] = make_float2(x[0], x[1]);
            rows[M + n] = make_float2(x[2], x[3]);
        }
        __syncthreads();
        fft_dif_rows<2>(rows, tws, m);
        for (int k = tid; k < 2 * M; k += nt) {
            const float2 y = c_mul(rows[k], spec[k & (M - 1)]);
            rows[k] = make_float2(y.x, -y.y);
        }
        __syncthreads();
        fft_dit_rows<2>(rows, tws, m);
        // out = conj(FFT(conj Y)): even rows the real part, odd rows minus
        // the imaginary part
        for (int e = 0; e < 4; ++e) {
            if (r0 + e >= nrows) break;
            float* o = out + (size_t)(r0 + e) * Nu;
            const float2* b = rows + (e >> 1) * M;
            for (int n = tid; n < Nu; n += nt) {
                const float2 v = b[n];
                o[n] = (e & 1) ? -v.y : v.x;
            }
        }
        __syncthreads();
    }
}

}  // namespace xr
