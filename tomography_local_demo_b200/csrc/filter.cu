// Projection ingest + FDK/FBP row filter, writing into the filtered-projection ring.
//
// Reference semantics (minirecast):
//   ramp_response    recon.py:34-55   spectrum H of the Kak & Slaney ramp kernel (host, FP64)
//   filter_rows      recon.py:58-64   rfft(n=N) * H[:N/2+1] -> irfft -> crop to C
//   fdk_filter_block recon.py:85-104  cosine pre-weight w = SDD / sqrt(SDD^2 + a^2 + b^2)
//   flexray.py:111-116, 174-184 / hdf5.py:24-31, 73-78: mean binning, (P-D)*gain,
//                    clip at 1e-3, -log (raw uint16 ingest)
//
// Design: one CTA filters 2*FPC rows of one view. Two real rows share one complex FFT
// (z = x1 + i x2): H is real and even, so H*Z transforms back to y1 + i y2 with no
// unpacking. The inverse FFT is a forward FFT of the conjugate. Radix-4 Stockham
// passes (plus one radix-2 pass for odd log2 N) ping-pong between two shared buffers;
// twiddles come from a caller-supplied FP64-accurate table through the read-only path.
#include "mr_common.cuh"

namespace mr {

struct Filter2Args {
    const float* block;
    const uint16_t* raw;
    long long s_view, s_row;
    int bin, flip;
    const float* dark;
    const float* gain;
    const mr_filter_view* views;
    const float* H;
    const float2* tw;
    void* ring;
    int dtype, rows, cols, pitch;
    long long slot_stride;
    int k;
};
template <bool RAW>
int launch_fft_filter_any(const Filter2Args& A, int log2n, cudaStream_t st);

constexpr int FLT_THREADS = 256;

struct FilterArgs {
    // input
    const float* block;          // f32 mode
    const uint16_t* raw;         // u16 mode
    long long s_view, s_row;
    int bin, flip;
    const float* dark;
    const float* gain;
    // per view
    const mr_filter_view* views;
    // filter tables
    const float* H;
    const float2* tw;
    // output ring
    void* ring;
    int dtype, rows, cols, pitch;
    long long slot_stride;
};

template <int LOG2N, int FPC>
__device__ __forceinline__ float2* fft_forward(float2* in, float2* out, const float2* __restrict__ tw) {
    constexpr int N = 1 << LOG2N;
    constexpr int NQ = N / 4;
#pragma unroll 1
    for (int s = 0; s < LOG2N / 2; ++s) {
        const int lns = 2 * s;
        const int Ns = 1 << lns;
        for (int it = threadIdx.x; it < FPC * NQ; it += FLT_THREADS) {
            const int f = it / NQ;
            const int j = it & (NQ - 1);
            const float2* x = in + f * N;
            float2* y = out + f * N;
            const int k = j & (Ns - 1);
            float2 v0 = x[j], v1 = x[j + NQ], v2 = x[j + 2 * NQ], v3 = x[j + 3 * NQ];
            if (s > 0) {
                const int step = k << (LOG2N - 2 - lns);
                v1 = cmul(v1, __ldg(tw + step));
                v2 = cmul(v2, __ldg(tw + 2 * step));
                v3 = cmul(v3, __ldg(tw + 3 * step));
            }
            const float2 a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3);
            const float2 d = csub(v1, v3);
            const float2 a3 = make_float2(d.y, -d.x);  // -i * (v1 - v3)
            const int base = ((j >> lns) << (lns + 2)) + k;
            y[base] = cadd(a0, a2);
            y[base + Ns] = cadd(a1, a3);
            y[base + 2 * Ns] = csub(a0, a2);
            y[base + 3 * Ns] = csub(a1, a3);
        }
        __syncthreads();
        float2* tmp = in; in = out; out = tmp;
    }
    if (LOG2N & 1) {
        constexpr int NH = N / 2;
        for (int it = threadIdx.x; it < FPC * NH; it += FLT_THREADS) {
            const int f = it / NH;
            const int j = it & (NH - 1);
            const float2* x = in + f * N;
            float2* y = out + f * N;
            const float2 v0 = x[j];
            const float2 v1 = cmul(x[j + NH], __ldg(tw + j));
            y[j] = cadd(v0, v1);
            y[j + NH] = csub(v0, v1);
        }
        __syncthreads();
        float2* tmp = in; in = out; out = tmp;
    }
    return in;
}

template <bool RAW>
__device__ __forceinline__ float load_x(const FilterArgs& A, int v, int r, int c) {
    if (!RAW) return __ldg(A.block + (long long)v * A.s_view + (long long)r * A.s_row + c);
    const int b = A.bin;
    const int rr = A.flip ? (A.rows - 1 - r) : r;
    const uint16_t* p = A.raw + (long long)v * A.s_view + (long long)rr * b * A.s_row + (long long)c * b;
    float s = 0.f;
    for (int dy = 0; dy < b; ++dy)
        for (int dx = 0; dx < b; ++dx) s += (float)__ldg(p + (long long)dy * A.s_row + dx);
    const float mean = __fdiv_rn(s, (float)(b * b));
    const int pix = r * A.cols + c;
    const float t = (mean - __ldg(A.dark + pix)) * __ldg(A.gain + pix);
    return -logf(fmaxf(t, 1e-3f));
}

__device__ __forceinline__ float fdk_weight(const mr_filter_view& fv, int r, int c) {
    if (fv.sdd == 0.f) return 1.f;
    const float a = fmaf((float)c, fv.da, fv.a0);
    const float b = fmaf((float)r, fv.db, fv.b0);
    return fv.sdd * rsqrtf(fmaf(fv.sdd, fv.sdd, fmaf(a, a, b * b)));
}

template <int LOG2N, int FPC, bool RAW>
__global__ void __launch_bounds__(FLT_THREADS) filter_kernel(FilterArgs A) {
    extern __shared__ float2 smem[];
    constexpr int N = 1 << LOG2N;
    float2* b0 = smem;
    float2* b1 = smem + FPC * N;
    const int v = blockIdx.y;
    const int row0 = blockIdx.x * (2 * FPC);
    const mr_filter_view fv = A.views[v];
    const int R = A.rows, C = A.cols;

    for (int it = threadIdx.x; it < FPC * N; it += FLT_THREADS) {
        const int f = it >> LOG2N, c = it & (N - 1);
        const int r = row0 + 2 * f;
        float re = 0.f, im = 0.f;
        if (c < C) {
            if (r < R) re = load_x<RAW>(A, v, r, c) * fdk_weight(fv, r, c);
            if (r + 1 < R) im = load_x<RAW>(A, v, r + 1, c) * fdk_weight(fv, r + 1, c);
        }
        b0[it] = make_float2(re, im);
    }
    __syncthreads();
    float2* spec = fft_forward<LOG2N, FPC>(b0, b1, A.tw);
    const float g = fv.gain * fv.out_scale;
    for (int it = threadIdx.x; it < FPC * N; it += FLT_THREADS) {
        const float h = __ldg(A.H + (it & (N - 1))) * g;
        const float2 z = spec[it];
        spec[it] = make_float2(z.x * h, -z.y * h);  // conj(H Z): inverse via a forward FFT
    }
    __syncthreads();
    float2* res = fft_forward<LOG2N, FPC>(spec, spec == b0 ? b1 : b0, A.tw);

    const int slot = fv.slot;
    for (int f = 0; f < FPC; ++f) {
        const int r = row0 + 2 * f;
        if (r >= R) break;
        const float2* z = res + f * N;
        for (int c = threadIdx.x; c < A.pitch; c += FLT_THREADS) {
            const float2 val = c < C ? z[c] : make_float2(0.f, 0.f);
            const long long o = (long long)slot * A.slot_stride + (long long)r * A.pitch + c;
            switch (A.dtype) {
                case MR_F32:
                    st_elem(static_cast<float*>(A.ring) + o, val.x);
                    if (r + 1 < R) st_elem(static_cast<float*>(A.ring) + o + A.pitch, -val.y);
                    break;
                case MR_BF16:
                    st_elem(static_cast<__nv_bfloat16*>(A.ring) + o, val.x);
                    if (r + 1 < R) st_elem(static_cast<__nv_bfloat16*>(A.ring) + o + A.pitch, -val.y);
                    break;
                default:
                    st_elem(static_cast<__half*>(A.ring) + o, val.x);
                    if (r + 1 < R) st_elem(static_cast<__half*>(A.ring) + o + A.pitch, -val.y);
                    break;
            }
        }
    }
}

constexpr int fpc_for(int log2n) {
    return log2n >= 12 ? 1 : ((4096 >> log2n) > 16 ? 16 : (4096 >> log2n));
}

template <int LOG2N, bool RAW>
static int launch_filter_n(const FilterArgs& A, int k, cudaStream_t st) {
    constexpr int FPC = fpc_for(LOG2N);
    constexpr int N = 1 << LOG2N;
    const size_t smem = 2ull * FPC * N * sizeof(float2);
    auto kern = filter_kernel<LOG2N, FPC, RAW>;
    MR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid((A.rows + 2 * FPC - 1) / (2 * FPC), k);
    kern<<<grid, FLT_THREADS, smem, st>>>(A);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

template <bool RAW>
static int launch_filter(const FilterArgs& A, int log2n, int k, cudaStream_t st) {
    if (log2n >= 5 && log2n <= 13) {            // register-resident FFT kernel
        Filter2Args B{A.block, A.raw, A.s_view, A.s_row, A.bin, A.flip, A.dark, A.gain, A.views, A.H,
                      A.tw, A.ring, A.dtype, A.rows, A.cols, A.pitch, A.slot_stride, k};
        return launch_fft_filter_any<RAW>(B, log2n, st);
    }
    switch (log2n) {
        case 4: return launch_filter_n<4, RAW>(A, k, st);
        case 5: return launch_filter_n<5, RAW>(A, k, st);
        case 6: return launch_filter_n<6, RAW>(A, k, st);
        case 7: return launch_filter_n<7, RAW>(A, k, st);
        case 8: return launch_filter_n<8, RAW>(A, k, st);
        case 9: return launch_filter_n<9, RAW>(A, k, st);
        case 10: return launch_filter_n<10, RAW>(A, k, st);
        case 11: return launch_filter_n<11, RAW>(A, k, st);
        case 12: return launch_filter_n<12, RAW>(A, k, st);
        case 13: return launch_filter_n<13, RAW>(A, k, st);
        default: return MR_ERR_UNSUPPORTED;
    }
}

static int check_common(const mr_ring* ring, int32_t k, const mr_filter_view* views,
                        const float* H, const float* tw, int32_t log2n) {
    if (!ring || !ring->data || !views || !H || !tw || k < 0) return MR_ERR_INVALID;
    if (ring->rows <= 0 || ring->cols <= 0 || ring->col_pitch < ring->cols) return MR_ERR_INVALID;
    if (ring->slot_stride < (int64_t)ring->rows * ring->col_pitch) return MR_ERR_INVALID;
    if (ring->dtype != MR_F32 && ring->dtype != MR_BF16 && ring->dtype != MR_F16) return MR_ERR_INVALID;
    if (log2n < 1 || log2n > 30 || (1LL << log2n) < 2LL * ring->cols) return MR_ERR_INVALID;
    return MR_OK;
}

static void fill_ring(FilterArgs& A, const mr_ring* ring, const mr_filter_view* views,
                      const float* H, const float* tw) {
    A.views = views;
    A.H = H;
    A.tw = reinterpret_cast<const float2*>(tw);
    A.ring = ring->data;
    A.dtype = ring->dtype;
    A.rows = ring->rows;
    A.cols = ring->cols;
    A.pitch = ring->col_pitch;
    A.slot_stride = ring->slot_stride;
}

}  // namespace mr

extern "C" int mr_filter_f32(const float* block, int64_t s_view, int64_t s_row, int32_t k,
                             const mr_filter_view* views, const float* H, const float* tw,
                             int32_t log2n, const mr_ring* ring, void* stream) {
    int rc = mr::check_common(ring, k, views, H, tw, log2n);
    if (rc != MR_OK) return rc;
    if (!block) return MR_ERR_INVALID;
    if (k == 0) return MR_OK;
    mr::FilterArgs A{};
    A.block = block;
    A.s_view = s_view;
    A.s_row = s_row;
    A.bin = 1;
    mr::fill_ring(A, ring, views, H, tw);
    return mr::launch_filter<false>(A, log2n, k, static_cast<cudaStream_t>(stream));
}

extern "C" int mr_ingest_u16(const uint16_t* raw, int64_t s_view, int64_t s_row, int32_t bin,
                             int32_t flip_rows, const float* dark, const float* gain, int32_t k,
                             const mr_filter_view* views, const float* H, const float* tw,
                             int32_t log2n, const mr_ring* ring, void* stream) {
    int rc = mr::check_common(ring, k, views, H, tw, log2n);
    if (rc != MR_OK) return rc;
    if (!raw || !dark || !gain || bin < 1 || bin > 16) return MR_ERR_INVALID;
    if (s_row < (int64_t)ring->cols * bin) return MR_ERR_INVALID;
    if (k == 0) return MR_OK;
    mr::FilterArgs A{};
    A.raw = raw;
    A.s_view = s_view;
    A.s_row = s_row;
    A.bin = bin;
    A.flip = flip_rows ? 1 : 0;
    A.dark = dark;
    A.gain = gain;
    mr::fill_ring(A, ring, views, H, tw);
    return mr::launch_filter<true>(A, log2n, k, static_cast<cudaStream_t>(stream));
}
