// Histogram-entropy score of trial slices for the rotation-centre search.
//
// minirecast recon.py:498-519 (estimate_cor): for every trial image,
//   hist, _ = np.histogram(img[img != 0], bins=128); p = hist[hist > 0] / max(hist.sum(), 1)
//   score = sum(p * log(p))              (= -entropy; the best shift maximises it)
// Per image: FP64 min/max of the non-zero pixels, a shared-memory histogram with
// numpy's uniform-bin rule (index = floor(((x - lo) / (hi - lo)) * bins), then corrected
// against the FP64 linspace edges, the top edge inclusive), and the FP64 sum.
#include <cooperative_groups.h>

#include "mr_common.cuh"

namespace cg = cooperative_groups;

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

// A cluster of ENT_CLUSTER CTAs per image, each over a contiguous share of its pixels: the
// min / max partials and the integer histograms are combined through distributed shared
// memory (exact), and rank 0 forms the score with the same thread / bin split a single
// CTA would use, so the scores do not depend on the cluster size.
constexpr int ENT_CLUSTER = 8;

__global__ void __launch_bounds__(ENT_THREADS, 2)
entropy_kernel(const float* __restrict__ imgs, long long stride, int n_pix, int bins, double* scores) {
    __shared__ double s_min[ENT_THREADS / 32], s_max[ENT_THREADS / 32];
    __shared__ unsigned int hist[ENT_MAX_BINS];
    __shared__ double s_lo, s_hi, s_red[ENT_THREADS / 32], s_part[2];
    __shared__ unsigned int s_cnt;
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank(), csize = (int)cluster.num_blocks();
    const int image = blockIdx.x / csize;
    const float* img = imgs + (long long)image * stride;
    const int p0 = (int)(((long long)n_pix * crank) / csize), p1 = (int)(((long long)n_pix * (crank + 1)) / csize);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    double mn = 1e308, mx = -1e308;
    for (int i = p0 + tid; i < p1; i += ENT_THREADS) {
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
        s_part[0] = a;
        s_part[1] = b;
    }
    cluster.sync();
    if (tid == 0) {
        double a = 1e308, b = -1e308;
        for (int r = 0; r < csize; ++r) {
            const double* pr = cluster.map_shared_rank(s_part, r);
            a = fmin(a, pr[0]);
            b = fmax(b, pr[1]);
        }
        if (a > b) { a = 0.0; b = 1.0; }               // no non-zero pixel: empty histogram
        if (a == b) { a -= 0.5; b += 0.5; }            // numpy widens a degenerate range
        s_lo = a; s_hi = b;
    }
    __syncthreads();
    const double lo = s_lo, hi = s_hi;
    const double denom = hi - lo;
    unsigned int cnt = 0;
    for (int i = p0 + tid; i < p1; i += ENT_THREADS) {
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
    cluster.sync();                                     // every share's histogram is complete
    if (crank == 0) {
        for (int b = tid; b < bins; b += ENT_THREADS) {
            unsigned int h = hist[b];
            for (int r = 1; r < csize; ++r) h += cluster.map_shared_rank(hist, r)[b];
            hist[b] = h;
        }
        if (tid == 0) {
            unsigned int c = s_cnt;
            for (int r = 1; r < csize; ++r) c += *cluster.map_shared_rank(&s_cnt, r);
            s_cnt = c;
        }
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
            double sum = 0.0;
            for (int w = 0; w < ENT_THREADS / 32; ++w) sum += s_red[w];
            scores[image] = sum;
        }
    }
    cluster.sync();                                     // the histograms stay alive until read
}

}  // namespace mr

extern "C" int mr_slice_entropy(const float* imgs, int32_t n_imgs, int64_t stride, int32_t n_pix,
                                int32_t bins, double* scores, void* stream) {
    if (!imgs || !scores || n_imgs < 0 || n_pix < 0 || bins < 1 || bins > mr::ENT_MAX_BINS) return MR_ERR_INVALID;
    if (stride < n_pix || n_imgs > 2147483647) return MR_ERR_INVALID;
    if (n_imgs == 0) return MR_OK;
    if ((long long)n_imgs * mr::ENT_CLUSTER > 2147483647LL) return MR_ERR_INVALID;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n_imgs * mr::ENT_CLUSTER));
    cfg.blockDim = dim3(mr::ENT_THREADS);
    cfg.stream = static_cast<cudaStream_t>(stream);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = mr::ENT_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MR_CUDA_TRY(cudaLaunchKernelEx(&cfg, mr::entropy_kernel, imgs, (long long)stride, n_pix, bins, scores));
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
