// Histogram-entropy score of trial slices for the rotation-centre search.
//
// minirecast recon.py:498-519 (estimate_cor): for every trial image,
//   hist, _ = np.histogram(img[img != 0], bins=128); p = hist[hist > 0] / max(hist.sum(), 1)
//   score = sum(p * log(p))              (= -entropy; the best shift maximises it)
// One CTA per image: FP64 min/max of the non-zero pixels, a shared-memory histogram with
// numpy's uniform-bin rule (index = floor(((x - lo) / (hi - lo)) * bins), then corrected
// against the FP64 linspace edges, the top edge inclusive), and the FP64 sum.
#include "mr_common.cuh"

namespace mr {

constexpr int ENT_THREADS = 512;
constexpr int ENT_MAX_BINS = 1024;

__device__ __forceinline__ double edge(double lo, double hi, int b, int bins) {
    // np.linspace(lo, hi, bins + 1): (b * step) + lo, each step rounded on its own (no FMA
    // contraction), the last edge exactly hi
    if (b >= bins) return hi;
    const double step = __ddiv_rn(__dsub_rn(hi, lo), (double)bins);
    return __dadd_rn(__dmul_rn((double)b, step), lo);
}

__global__ void __launch_bounds__(ENT_THREADS)
entropy_kernel(const float* __restrict__ imgs, long long stride, int n_pix, int bins, double* scores) {
    __shared__ double s_min[ENT_THREADS / 32], s_max[ENT_THREADS / 32];
    __shared__ unsigned int hist[ENT_MAX_BINS];
    __shared__ double s_lo, s_hi, s_red[ENT_THREADS / 32];
    __shared__ unsigned int s_cnt;
    const float* img = imgs + (long long)blockIdx.x * stride;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    double mn = 1e308, mx = -1e308;
    for (int i = tid; i < n_pix; i += ENT_THREADS) {
        const float v = img[i];
        if (v != 0.f) {
            mn = fmin(mn, (double)v);
            mx = fmax(mx, (double)v);
        }
    }
    for (int o = 16; o; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) { s_min[warp] = mn; s_max[warp] = mx; }
    for (int b = tid; b < bins; b += ENT_THREADS) hist[b] = 0u;
    if (tid == 0) s_cnt = 0u;
    __syncthreads();
    if (tid == 0) {
        double a = 1e308, b = -1e308;
        for (int w = 0; w < ENT_THREADS / 32; ++w) { a = fmin(a, s_min[w]); b = fmax(b, s_max[w]); }
        if (a > b) { a = 0.0; b = 1.0; }               // no non-zero pixel: empty histogram
        if (a == b) { a -= 0.5; b += 0.5; }            // numpy widens a degenerate range
        s_lo = a; s_hi = b;
    }
    __syncthreads();
    const double lo = s_lo, hi = s_hi;
    const double denom = hi - lo;
    unsigned int cnt = 0;
    for (int i = tid; i < n_pix; i += ENT_THREADS) {
        const float vf = img[i];
        if (vf == 0.f) continue;
        const double v = vf;
        int k = (int)__dmul_rn(__ddiv_rn(__dsub_rn(v, lo), denom), (double)bins);   // ((x - lo) / (hi - lo)) * bins
        if (k >= bins) k = bins - 1;
        if (k < 0) k = 0;
        if (v < edge(lo, hi, k, bins)) --k;
        else if (k != bins - 1 && v >= edge(lo, hi, k + 1, bins)) ++k;
        k = k < 0 ? 0 : (k >= bins ? bins - 1 : k);
        atomicAdd(&hist[k], 1u);
        ++cnt;
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) atomicAdd(&s_cnt, cnt);
    __syncthreads();
    const double total = s_cnt > 0 ? (double)s_cnt : 1.0;
    double acc = 0.0;
    for (int b = tid; b < bins; b += ENT_THREADS) {
        if (hist[b]) {
            const double p = hist[b] / total;
            acc += p * log(p);
        }
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < ENT_THREADS / 32; ++w) s += s_red[w];
        scores[blockIdx.x] = s;
    }
}

}  // namespace mr

extern "C" int mr_slice_entropy(const float* imgs, int32_t n_imgs, int64_t stride, int32_t n_pix,
                                int32_t bins, double* scores, void* stream) {
    if (!imgs || !scores || n_imgs < 0 || n_pix < 0 || bins < 1 || bins > mr::ENT_MAX_BINS) return MR_ERR_INVALID;
    if (stride < n_pix || n_imgs > 2147483647) return MR_ERR_INVALID;
    if (n_imgs == 0) return MR_OK;
    mr::entropy_kernel<<<n_imgs, mr::ENT_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        imgs, (long long)stride, n_pix, bins, scores);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
