// Projection pre-processing on arrival (minirecast preprocess.py), block layout
// [rows, k, cols] (ASTRA) in and out, FP32.
//
//   rotate_projections preprocess.py:31-56: out(r,c) = bilinear(in, rs, cs), zero
//       outside, rs = cos t * rr + sin t * cc + (R-1)/2, cs = -sin t * rr + cos t * cc + (C-1)/2
//   gaussian_blur      preprocess.py:8-28: per axis, edge padding by pad = ceil(3 sigma),
//       circular convolution of length N = n + 2 pad with g = irfft(exp(-2 (pi f sigma)^2)),
//       crop. The caller passes g[0..K] (g is even; |m| > K contributes < 1e-20).
#include "mr_common.cuh"

namespace mr {

__global__ void rotate_kernel(const float* __restrict__ in, float* __restrict__ out, int R, int A,
                              int C, float ct, float st) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    const int a = blockIdx.z;
    if (c >= C) return;
    const float rr = (float)r - 0.5f * (float)(R - 1);
    const float cc = (float)c - 0.5f * (float)(C - 1);
    const float rs = fmaf(ct, rr, st * cc) + 0.5f * (float)(R - 1);
    const float cs = fmaf(-st, rr, ct * cc) + 0.5f * (float)(C - 1);
    const float r0f = floorf(rs), c0f = floorf(cs);
    const float fr = rs - r0f, fc = cs - c0f;
    const int r0 = (int)r0f, c0 = (int)c0f;
    const long long srow = (long long)A * C;
    float acc = 0.f;
#pragma unroll
    for (int dr = 0; dr < 2; ++dr) {
#pragma unroll
        for (int dc = 0; dc < 2; ++dc) {
            const int ri = r0 + dr, ci = c0 + dc;
            if ((unsigned)ri < (unsigned)R && (unsigned)ci < (unsigned)C) {
                const float w = (dr ? fr : 1.f - fr) * (dc ? fc : 1.f - fc);
                acc = fmaf(w, __ldg(in + ri * srow + (long long)a * C + ci), acc);
            }
        }
    }
    out[r * srow + (long long)a * C + c] = acc;
}

// One axis of the edge-padded circular Gaussian: along rows (axis 0) or cols (axis 2).
__global__ void gauss_axis_kernel(const float* __restrict__ in, float* __restrict__ out, int R, int A,
                                  int C, int axis, int pad, const float* __restrict__ g, int K) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    const int a = blockIdx.z;
    if (c >= C) return;
    const long long srow = (long long)A * C;
    const int n = axis == 0 ? R : C;
    const int i = axis == 0 ? r : c;
    const int Np = n + 2 * pad;
    const float* base = axis == 0 ? in + (long long)a * C + c : in + r * srow + (long long)a * C;
    const long long step = axis == 0 ? srow : 1;
    float acc = 0.f;
    for (int m = -K; m <= K; ++m) {
        int t = i + pad - m;                 // index into the padded signal, circular
        t %= Np;
        if (t < 0) t += Np;
        int src = t - pad;                   // edge padding
        src = src < 0 ? 0 : (src >= n ? n - 1 : src);
        acc = fmaf(__ldg(g + (m < 0 ? -m : m)), __ldg(base + src * step), acc);
    }
    out[r * srow + (long long)a * C + c] = acc;
}

}  // namespace mr

extern "C" int mr_rotate_f32(const float* in, float* out, int32_t rows, int32_t k, int32_t cols,
                             double degrees, void* stream) {
    if (!in || !out || rows <= 0 || cols <= 0 || k < 0 || in == out) return MR_ERR_INVALID;
    if (k == 0) return MR_OK;
    const double t = degrees * 3.14159265358979323846 / 180.0;
    const dim3 block(128);
    const dim3 grid((cols + 127) / 128, rows, k);
    if (k > 65535 || rows > 65535) return MR_ERR_INVALID;
    mr::rotate_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        in, out, rows, k, cols, (float)cos(t), (float)sin(t));
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

extern "C" int mr_gaussian_axis_f32(const float* in, float* out, int32_t rows, int32_t k,
                                    int32_t cols, int32_t axis, int32_t pad, const float* taps,
                                    int32_t n_taps, void* stream) {
    if (!in || !out || !taps || rows <= 0 || cols <= 0 || k < 0 || in == out) return MR_ERR_INVALID;
    if ((axis != 0 && axis != 2) || pad < 0 || n_taps < 1) return MR_ERR_INVALID;
    if (k == 0) return MR_OK;
    if (k > 65535 || rows > 65535) return MR_ERR_INVALID;
    const dim3 block(128);
    const dim3 grid((cols + 127) / 128, rows, k);
    mr::gauss_axis_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        in, out, rows, k, cols, axis, pad, taps, n_taps - 1);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
