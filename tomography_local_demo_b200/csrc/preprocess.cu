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

// The same axis convolution organised for the SM. For small sigma the taps reach about half
// the padded length (the spectrum is cut at Nyquist), so a direct loop costs ~n/2 taps per
// output. A block takes L lines (rows along axis 2, columns along axis 0) and TO outputs of
// each: it stages the stretch of the edge-padded, periodically extended line those outputs
// read into shared memory once, then every thread computes 8 consecutive outputs of one
// line, 8 taps at a time: 15 staged values in registers serve the 64 products of a block of
// taps. The taps are padded in front with zeros to a multiple of 8 (m from K - 8 nb + 1);
// those add 0 * x to a zero sum, exactly, so each output is the same FMA chain over
// m = -K .. K as in gauss_axis_kernel and the results are identical.
constexpr int GS_THREADS = 256;
constexpr int GS_RUN = 8;                       // consecutive outputs per thread = taps per block

template <int L, int LP>
__global__ void __launch_bounds__(GS_THREADS)
gauss_lines_kernel(const float* __restrict__ in, float* __restrict__ out, int R, int A, int C, int axis,
                   int pad, const float* __restrict__ g, int K, int TO) {
    extern __shared__ float gsm[];
    const int nb = (2 * K + 1 + GS_RUN - 1) / GS_RUN;           // blocks of 8 taps
    const int m0 = K - GS_RUN * nb + 1;                        // first (zero-padded) tap
    const int T = TO + GS_RUN * nb;             // staged positions per line
    float* taps = gsm;                          // [8 nb]: tap m0 + i
    float* ext = gsm + GS_RUN * nb;             // [T][LP]
    const long long srow = (long long)A * C;
    const int n = axis == 0 ? R : C;
    const int Np = n + 2 * pad;
    const long long n_lines = axis == 0 ? (long long)A * C : (long long)R * A;
    const long long line0 = (long long)blockIdx.x * L;
    const int i0 = blockIdx.y * TO;
    const long long step = axis == 0 ? srow : 1;
    auto line_base = [&](long long line) -> long long {
        if (axis == 0) return line;                                     // a * C + c
        const long long r = line / A, a = line - r * A;
        return r * srow + a * C;
    };
    for (int i = threadIdx.x; i < GS_RUN * nb; i += GS_THREADS) {
        const int m = m0 + i;
        taps[i] = m < -K ? 0.f : __ldg(g + (m < 0 ? -m : m));
    }
    // staged position t holds padded position i0 + pad - K + t; output o at tap m reads t = o + K - m
    const int nl = (int)min((long long)L, n_lines - line0);
    for (int e = threadIdx.x; e < L * T; e += GS_THREADS) {
        int l, t;
        if (axis == 0) { l = e % L; t = e / L; }                        // neighbouring columns
        else { l = e / T; t = e - (e / T) * T; }                        // along one row
        float v = 0.f;
        if (l < nl) {
            int u = i0 + pad - K + t;                                   // padded position
            u %= Np;
            if (u < 0) u += Np;                                         // circular
            int src = u - pad;                                          // edge padding
            src = src < 0 ? 0 : (src >= n ? n - 1 : src);
            v = __ldg(in + line_base(line0 + l) + src * step);
        }
        ext[t * LP + l] = v;
    }
    __syncthreads();
    const int groups = (TO + GS_RUN - 1) / GS_RUN;
    for (int task = threadIdx.x; task < L * groups; task += GS_THREADS) {
        const int l = task % L, q = task / L;
        const int o0 = q * GS_RUN;                                      // first output (block-local)
        if (l >= nl || i0 + o0 >= n) continue;
        float acc[GS_RUN];
#pragma unroll
        for (int j = 0; j < GS_RUN; ++j) acc[j] = 0.f;
        for (int b = 0; b < nb; ++b) {
            // taps m = mb + u (u < 8) of outputs o0 + j read t = o0 + j + K - mb - u
            const int base = o0 + K - (m0 + GS_RUN * b) - (GS_RUN - 1);
            float w[2 * GS_RUN - 1];
#pragma unroll
            for (int k = 0; k < 2 * GS_RUN - 1; ++k) w[k] = ext[(base + k) * LP + l];
#pragma unroll
            for (int u = 0; u < GS_RUN; ++u) {
                const float gm = taps[GS_RUN * b + u];
#pragma unroll
                for (int j = 0; j < GS_RUN; ++j) acc[j] = fmaf(gm, w[j - u + GS_RUN - 1], acc[j]);
            }
        }
        const long long lb = line_base(line0 + l);
#pragma unroll
        for (int j = 0; j < GS_RUN; ++j) {
            const int i = i0 + o0 + j;
            if (i < n && o0 + j < TO) out[lb + (long long)i * step] = acc[j];
        }
    }
}

// LP: the staged line stride (L + 1, or 18 for 16 lines: the two half-warps of a warp,
// 8 staged positions apart, then fall on opposite halves of the banks)
template <int LP>
static size_t gauss_lines_smem(int K, int TO) {
    const int nb = (2 * K + 1 + GS_RUN - 1) / GS_RUN;
    return ((size_t)(TO + GS_RUN * nb) * LP + (size_t)GS_RUN * nb) * sizeof(float);
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
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int K = n_taps - 1;
    const int n = axis == 0 ? rows : cols;
    const long long n_lines = axis == 0 ? (long long)k * cols : (long long)rows * k;
    constexpr size_t kSmemMax = 200 * 1024;
    // whole lines per block (16 lines: every input staged about twice, the periodic
    // extension) where they fit, else 8 lines x 256 outputs
    const int whole = (n + mr::GS_RUN - 1) / mr::GS_RUN * mr::GS_RUN;
    if (K <= n + 2 * pad && mr::gauss_lines_smem<18>(K, whole) <= kSmemMax) {
        const size_t smem = mr::gauss_lines_smem<18>(K, whole);
        MR_CUDA_TRY(cudaFuncSetAttribute(mr::gauss_lines_kernel<16, 18>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const dim3 grid((unsigned)((n_lines + 15) / 16), 1);
        mr::gauss_lines_kernel<16, 18><<<grid, mr::GS_THREADS, smem, st>>>(in, out, rows, k, cols, axis, pad, taps,
                                                                            K, whole);
    } else if (K <= n + 2 * pad && mr::gauss_lines_smem<9>(K, 256) <= kSmemMax) {
        const size_t smem = mr::gauss_lines_smem<9>(K, 256);
        MR_CUDA_TRY(cudaFuncSetAttribute(mr::gauss_lines_kernel<8, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
        const dim3 grid((unsigned)((n_lines + 7) / 8), (unsigned)((n + 255) / 256));
        mr::gauss_lines_kernel<8, 9><<<grid, mr::GS_THREADS, smem, st>>>(in, out, rows, k, cols, axis, pad, taps, K,
                                                                          256);
    } else {
        const dim3 block(128);
        const dim3 grid((cols + 127) / 128, rows, k);
        mr::gauss_axis_kernel<<<grid, block, 0, st>>>(in, out, rows, k, cols, axis, pad, taps, K);
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
