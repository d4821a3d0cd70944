// Volume consumers on the device: the Otsu threshold of minirecast model.py:18-29,
//   v = vol[vol != 0]; lo, hi = np.percentile(v, [0.1, 99.95])
//   hist, edges = np.histogram(np.clip(v, lo, hi), bins=bins, range=(lo, hi))
// reduced to three streaming passes over the volume (any number of voxels, FP32):
//   mr_volume_stats      count of non-zero voxels and NaNs, min / max order key
//   mr_volume_select     exact order statistics of the non-zero voxels (radix select on
//                        order-preserving keys, 11-bit digits below the bits that the
//                        smallest and largest key share: at most 3 passes)
//   mr_volume_histogram  numpy's uniform-bin histogram of the FP64-clipped values
// The percentile interpolation and the Otsu arithmetic over the bins stay on the host,
// in FP64 as the reference computes them.
//
// Every pass reads the voxels as float4 where aligned, and combines the increments of
// neighbouring lanes that fall in the same bin into one shared-memory atomic (voxels next
// to each other in memory mostly share a bin, which would otherwise serialise the warp on
// one address).
#include "mr_common.cuh"

namespace mr {

constexpr int VOL_THREADS = 256;
constexpr int VOL_MAX_RANKS = 4;
constexpr int VOL_MAX_BINS = 2048;
constexpr int VOL_RADIX = 11;                   // digit bits of one select pass
constexpr int VOL_DIGITS = 1 << VOL_RADIX;
constexpr uint32_t VOL_NONE = 0xffffffffu;
constexpr unsigned FULL = 0xffffffffu;

// Device workspace of the three entry points (zeroed by mr_volume_stats).
struct VolState {
    unsigned long long nonzero;             // voxels != 0 (NaNs included, as vol != 0 keeps them)
    unsigned long long nan;                 // NaN voxels
    unsigned int kmin, kmax;                // order keys of the smallest / largest non-NaN value != 0
    unsigned int prefix[VOL_MAX_RANKS];     // key bits found so far, per requested rank
    unsigned long long rank[VOL_MAX_RANKS]; // rank left inside the current prefix
    unsigned long long hist[VOL_MAX_RANKS][VOL_DIGITS];
};

// Order-preserving map of a float onto an unsigned key (negatives reversed below positives).
__device__ __forceinline__ uint32_t order_key(float x) {
    const uint32_t b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_value(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// hist[b] += 1 for every lane whose b != VOL_NONE; a run of equal b in consecutive lanes
// is one atomic of the run length. All 32 lanes of the warp call it.
__device__ __forceinline__ void warp_run_add(unsigned int* hist, uint32_t b, int lane) {
    const uint32_t prev = __shfl_up_sync(FULL, b, 1);
    const bool head = lane == 0 || prev != b;
    const uint32_t heads = __ballot_sync(FULL, head);
    if (head && b != VOL_NONE) {
        const uint32_t above = lane == 31 ? 0u : (heads & (0xffffffffu << (lane + 1)));
        const int next = above ? __ffs(above) - 1 : 32;
        atomicAdd(hist + b, (unsigned)(next - lane));
    }
}

// Visits every voxel once: aligned float4 body in warp-uniform steps of 4 loads per lane
// (fn receives 4 values per load slot and a validity flag, called by all lanes), then the
// unaligned head and the tail (fewer than 4 + 3 voxels) by warp 0 of block 0.
template <typename Fn>
__device__ __forceinline__ void for_each_voxel(const float* __restrict__ v, long long n, Fn&& fn) {
    const int lane = threadIdx.x & 31;
    long long head = (long long)((((uint32_t)(uintptr_t)v) & 15u) ? (16u - (((uint32_t)(uintptr_t)v) & 15u)) >> 2 : 0u);
    if (head > n) head = n;
    const float4* __restrict__ v4 = reinterpret_cast<const float4*>(v + head);
    const long long n4 = (n - head) >> 2;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    constexpr int U = 4;
    for (long long base = gw * 32 * U; base < n4; base += warps * 32 * U) {
        float4 q[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long i = base + u * 32 + lane;
            ok[u] = i < n4;
            q[u] = ok[u] ? __ldg(v4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            fn(q[u].x, ok[u]);
            fn(q[u].y, ok[u]);
            fn(q[u].z, ok[u]);
            fn(q[u].w, ok[u]);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < 32) {
        const long long t0 = head + (n4 << 2);             // tail: [t0, n), fewer than 4
        const long long i = lane < head ? lane : t0 + (lane - 4);
        const bool ok = lane < head || (lane >= 4 && lane < 8 && i < n);
        fn(ok ? v[i] : 0.f, ok);
    }
}

__global__ void __launch_bounds__(VOL_THREADS)
vol_stats_kernel(const float* __restrict__ v, long long n, VolState* st) {
    unsigned long long nz = 0, nan = 0;
    uint32_t kmin = 0xffffffffu, kmax = 0u;
    for_each_voxel(v, n, [&](float x, bool ok) {
        if (!ok) return;
        nz += (x != 0.f);
        nan += (x != x);
        if (x != 0.f && x == x) {
            const uint32_t k = order_key(x);
            kmin = min(kmin, k);
            kmax = max(kmax, k);
        }
    });
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        nz += __shfl_xor_sync(FULL, nz, o);
        nan += __shfl_xor_sync(FULL, nan, o);
        kmin = min(kmin, __shfl_xor_sync(FULL, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(FULL, kmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (nz) atomicAdd(&st->nonzero, nz);
        if (nan) atomicAdd(&st->nan, nan);
        if (kmin <= kmax) {
            atomicMin(&st->kmin, kmin);
            atomicMax(&st->kmax, kmax);
        }
    }
}

// One radix digit for every requested rank: voxels whose key matches the rank's prefix
// above the digit count into that rank's 2^width bins. shared = 1: all ranks still share
// their prefix, so one histogram serves them all. After the first pass a prefix covers a
// small part of the voxels, so a warp whose voxels match no prefix moves on after one vote.
__global__ void __launch_bounds__(VOL_THREADS)
vol_select_pass_kernel(const float* __restrict__ v, long long n, VolState* st, int n_ranks, int shared,
                       int shift, int width, uint32_t mask_hi) {
    __shared__ unsigned int h[VOL_MAX_RANKS][VOL_DIGITS];
    const int n_hist = shared ? 1 : n_ranks;
    for (int i = threadIdx.x; i < n_hist * VOL_DIGITS; i += blockDim.x) (&h[0][0])[i] = 0u;
    uint32_t pre[VOL_MAX_RANKS];
#pragma unroll
    for (int j = 0; j < VOL_MAX_RANKS; ++j) pre[j] = st->prefix[j] & mask_hi;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t dmask = (1u << width) - 1u;
    for_each_voxel(v, n, [&](float x, bool ok) {
        const bool live = ok && x != 0.f && x == x;
        const uint32_t k = order_key(x);
        const uint32_t hi = k & mask_hi;
        bool m[VOL_MAX_RANKS];
        bool any = false;
#pragma unroll
        for (int j = 0; j < VOL_MAX_RANKS; ++j) {
            m[j] = live && j < n_hist && hi == pre[j];
            any |= m[j];
        }
        if (!__any_sync(FULL, any)) return;                 // warp-uniform
        const uint32_t d = (k >> shift) & dmask;
#pragma unroll
        for (int j = 0; j < VOL_MAX_RANKS; ++j) {
            if (j < n_hist && __any_sync(FULL, m[j]))       // warp-uniform
                warp_run_add(h[j], m[j] ? d : VOL_NONE, lane);
        }
    });
    __syncthreads();
    for (int i = threadIdx.x; i < n_hist * VOL_DIGITS; i += blockDim.x) {
        const unsigned int c = (&h[0][0])[i];
        if (c) atomicAdd(&st->hist[i / VOL_DIGITS][i % VOL_DIGITS], (unsigned long long)c);
    }
}

// Picks each rank's digit from its histogram (exclusive prefix sums over the bins), narrows
// the rank, clears the histograms. One block of 256 threads, 8 bins per thread.
__global__ void __launch_bounds__(256) vol_select_pick_kernel(VolState* st, int n_ranks, int shared, int shift) {
    constexpr int PER = VOL_DIGITS / 256;
    __shared__ unsigned long long warp_tot[8];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int j = 0; j < n_ranks; ++j) {
        const unsigned long long* hj = st->hist[shared ? 0 : j] + t * PER;
        unsigned long long c = 0;
#pragma unroll
        for (int i = 0; i < PER; ++i) c += hj[i];
        unsigned long long incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        unsigned long long off = 0;
        for (int w = 0; w < warp; ++w) off += warp_tot[w];
        incl += off;
        unsigned long long excl = incl - c;
        const unsigned long long r = st->rank[j];
        __syncthreads();                    // every thread has read rank[j] and warp_tot
        if (c > 0 && excl <= r && r < incl) {
            int b = 0;
            for (; b < PER - 1 && excl + hj[b] <= r; ++b) excl += hj[b];
            st->prefix[j] |= (uint32_t)(t * PER + b) << shift;
            st->rank[j] = r - excl;
        }
        __syncthreads();
    }
    for (int i = t; i < VOL_MAX_RANKS * VOL_DIGITS; i += 256) (&st->hist[0][0])[i] = 0ull;
}

struct RankList {
    long long r[VOL_MAX_RANKS];
};

__global__ void vol_select_init_kernel(VolState* st, RankList ranks, int n_ranks, uint32_t prefix) {
    const int j = threadIdx.x;
    if (j < VOL_MAX_RANKS) {
        st->prefix[j] = prefix;
        st->rank[j] = j < n_ranks ? (unsigned long long)ranks.r[j] : 0ull;
    }
    for (int i = threadIdx.x; i < VOL_MAX_RANKS * VOL_DIGITS; i += blockDim.x) (&st->hist[0][0])[i] = 0ull;
}

__global__ void vol_select_out_kernel(const VolState* st, int n_ranks, float* out) {
    const int j = threadIdx.x;
    if (j < n_ranks) out[j] = key_value(st->prefix[j]);
}

// np.histogram(np.clip(v, lo, hi), bins, range) over the non-zero voxels, in FP32: a float
// x lies in bin k (edges[k] <= x < edges[k+1], FP64 edges = numpy's linspace, passed in)
// exactly when lb[k] <= x < lb[k+1], lb[i] = edges[i] rounded up to a float (the smallest
// float >= the edge); the top edge counts in the last bin. The clip is exact the same way:
// x < lo exactly when x < lo rounded up, x > hi exactly when x > hi rounded down, and those
// voxels take the bin of lo / hi. numpy's own rule (index from ((x - first) / (last -
// first)) * bins, corrected by one step against the same edges) lands in the same bin.
__global__ void __launch_bounds__(VOL_THREADS)
vol_histogram_kernel(const float* __restrict__ v, long long n, const double* __restrict__ edges, int bins,
                     double lo, double hi, unsigned long long* __restrict__ hist) {
    __shared__ unsigned int h[VOL_MAX_BINS];
    __shared__ float lb[VOL_MAX_BINS + 1];
    __shared__ int s_bin_lo, s_bin_hi;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) h[i] = 0u;
    for (int i = threadIdx.x; i <= bins; i += blockDim.x) lb[i] = __double2float_ru(edges[i]);
    if (threadIdx.x == 0) {
        // bins of the clip bounds themselves (lo, hi inside [edges[0], edges[bins]])
        int a = 0, b = bins - 1;
        while (a < bins - 1 && lo >= edges[a + 1]) ++a;
        while (b > 0 && hi < edges[b]) --b;
        s_bin_lo = a;
        s_bin_hi = b;
    }
    __syncthreads();
    const float lo_up = __double2float_ru(lo), hi_dn = __double2float_rd(hi);
    const float first = lb[0], scale = (float)bins / (lb[bins] - lb[0]);
    const int bin_lo = s_bin_lo, bin_hi = s_bin_hi;
    const int lane = threadIdx.x & 31;
    for_each_voxel(v, n, [&](float x, bool ok) {
        uint32_t b = VOL_NONE;
        if (ok && x != 0.f && x == x) {
            int k;
            if (x < lo_up) {
                k = bin_lo;
            } else if (x > hi_dn) {
                k = bin_hi;
            } else {
                const float f = (x - first) * scale;
                k = f >= (float)bins ? bins - 1 : (f > 0.f ? (int)f : 0);
                while (k > 0 && x < lb[k]) --k;
                while (k < bins - 1 && x >= lb[k + 1]) ++k;
            }
            b = (uint32_t)k;
        }
        warp_run_add(h, b, lane);
    });
    __syncthreads();
    for (int i = threadIdx.x; i < bins; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

static int vol_grid(int* blocks) {
    int dev = 0, sms = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *blocks = 4 * (sms > 0 ? sms : 1);
    return MR_OK;
}

}  // namespace mr

extern "C" int64_t mr_volume_workspace_bytes(void) { return (int64_t)sizeof(mr::VolState); }

extern "C" int mr_volume_stats(const float* vol, int64_t n, void* ws, uint64_t* stats_host, void* stream) {
    if (!ws || n < 0 || (n > 0 && !vol)) return MR_ERR_INVALID;
    if (((uintptr_t)vol & 3u) || ((uintptr_t)ws & 7u)) return MR_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mr::VolState* s = static_cast<mr::VolState*>(ws);
    MR_CUDA_TRY(cudaMemsetAsync(s, 0, sizeof(mr::VolState), st));
    MR_CUDA_TRY(cudaMemsetAsync(&s->kmin, 0xff, sizeof(unsigned int), st));
    int blocks = 0;
    const int rc = mr::vol_grid(&blocks);
    if (rc != MR_OK) return rc;
    if (n > 0) mr::vol_stats_kernel<<<blocks, mr::VOL_THREADS, 0, st>>>(vol, (long long)n, s);
    MR_CUDA_TRY(cudaGetLastError());
    if (stats_host) {
        // nonzero, nan, (kmin | kmax << 32): 24 bytes of the workspace head
        MR_CUDA_TRY(cudaMemcpyAsync(stats_host, s, 3 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        MR_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return MR_OK;
}

extern "C" int mr_volume_select(const float* vol, int64_t n, const int64_t* ranks, int32_t n_ranks,
                                uint32_t kmin, uint32_t kmax, void* ws, float* values_dev, void* stream) {
    if (!ws || !ranks || !values_dev || n <= 0 || !vol) return MR_ERR_INVALID;
    if (n_ranks < 1 || n_ranks > mr::VOL_MAX_RANKS || kmin > kmax) return MR_ERR_INVALID;
    mr::RankList rl = {};
    for (int j = 0; j < n_ranks; ++j) {
        if (ranks[j] < 0 || ranks[j] >= n) return MR_ERR_INVALID;
        rl.r[j] = (long long)ranks[j];
    }
    if (((uintptr_t)vol & 3u) || ((uintptr_t)ws & 7u)) return MR_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mr::VolState* s = static_cast<mr::VolState*>(ws);
    int blocks = 0;
    const int rc = mr::vol_grid(&blocks);
    if (rc != MR_OK) return rc;
    // bits [0, L) vary between the smallest and largest key; the bits above are known
    const int L = (kmin == kmax) ? 0 : 32 - __builtin_clz(kmin ^ kmax);
    const uint32_t known = L >= 32 ? 0u : ~((1u << L) - 1u);
    mr::vol_select_init_kernel<<<1, 256, 0, st>>>(s, rl, n_ranks, kmin & known);
    for (int top = L, pass = 0; top > 0; top -= mr::VOL_RADIX, ++pass) {
        const int shift = top > mr::VOL_RADIX ? top - mr::VOL_RADIX : 0;
        const int width = top - shift;
        const uint32_t mask_hi = top >= 32 ? 0u : ~((1u << top) - 1u);
        const int shared = pass == 0 ? 1 : 0;
        mr::vol_select_pass_kernel<<<blocks, mr::VOL_THREADS, 0, st>>>(vol, (long long)n, s, n_ranks, shared,
                                                                      shift, width, mask_hi);
        mr::vol_select_pick_kernel<<<1, 256, 0, st>>>(s, n_ranks, shared, shift);
    }
    mr::vol_select_out_kernel<<<1, 32, 0, st>>>(s, n_ranks, values_dev);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

extern "C" int mr_volume_histogram(const float* vol, int64_t n, const double* edges_dev, int32_t bins,
                                   double lo, double hi, uint64_t* hist_dev, void* stream) {
    if (!edges_dev || !hist_dev || n < 0 || (n > 0 && !vol)) return MR_ERR_INVALID;
    if (bins < 1 || bins > mr::VOL_MAX_BINS || !(lo <= hi)) return MR_ERR_INVALID;
    if (((uintptr_t)vol & 3u) || ((uintptr_t)edges_dev & 7u) || ((uintptr_t)hist_dev & 7u)) return MR_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // numpy widens an empty range by 0.5 on each side; the edges passed in already are
    double first = lo, last = hi;
    if (first == last) { first -= 0.5; last += 0.5; }
    const double scale = (double)bins / (last - first);
    if (!(scale > 0.0) || scale != scale || scale > 1.7976931348623157e308) return MR_ERR_INVALID;
    MR_CUDA_TRY(cudaMemsetAsync(hist_dev, 0, sizeof(uint64_t) * (size_t)bins, st));
    int blocks = 0;
    const int rc = mr::vol_grid(&blocks);
    if (rc != MR_OK) return rc;
    if (n > 0)
        mr::vol_histogram_kernel<<<blocks, mr::VOL_THREADS, 0, st>>>(
            vol, (long long)n, edges_dev, bins, lo, hi, reinterpret_cast<unsigned long long*>(hist_dev));
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
