// TMA-staged voxel-driven back-projection for regular grids (slices, windows, volumes).
//
// Same result as bp.cu (minirecast recon.py:156-219 semantics), different data path:
//   * per (tile, view) the CTA projects the tile's 4 corners (a planar tile maps to the
//     convex hull of its corners' projections) and derives the detector footprint;
//   * one thread issues cp.async.bulk.tensor 3D box loads (W cols x 8 rows, single CTA,
//     no multicast) of that footprint into a shared-memory stage; loads outside the
//     detector are zero-filled by the TMA unit, which is exactly the reference's
//     "bilinear taps outside [0,R)x[0,C) contribute 0";
//   * a warp-specialised ring of stages: one producer warp computes footprints and issues
//     the TMA loads, eight consumer warps back-project; full/empty mbarriers (bounded
//     waits) are the only synchronisation inside the view loop;
//   * the consumer loop is predicate-free: floor via a round-down FMA against a magic
//     constant (FMA pipe only), one unsigned clamp for memory safety, four LDS, lerps;
//   * footprints that miss the detector entirely are skipped (exactly zero), and the
//     rare footprints larger than a stage fall back to predicated global loads.
// Each warp covers compact 8 (j) x 4 (i) sample patches so its LDS gathers touch a small
// 2D patch (few bank conflicts) for any plane orientation.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cooperative_groups.h>
#include <mutex>
#include <type_traits>

#include "mr_common.cuh"

namespace cg = cooperative_groups;

namespace mr {

constexpr int ST_TI = 32, ST_TJ = 32;        // tile (samples) - same tiling as bp.cu
constexpr int ST_CONSUMERS = 8;               // consumer warps (one 32 x 32 tile)
constexpr int ST_THREADS = 32 * (ST_CONSUMERS + 1);   // + one producer warp
constexpr int ST_PPT = 4;                     // samples per consumer thread (rows i, i+2, i+4, i+6)
constexpr int ST_DI = 2;                      // row step between a thread's samples
constexpr int ST_BOX_H = 8;                   // rows per TMA box
constexpr int ST_CLUSTER = 4;                 // CTAs per tile, each a quarter of the views
constexpr float MAGIC = 12582912.0f;          // 1.5 * 2^23
constexpr int MAGIC_BITS = 0x4B400000;
#define kMagic2 make_float2(MAGIC, MAGIC)
#define kNeg2 make_float2(-1.f, -1.f)

template <typename T> struct StageGeom;
// Row widths (elements) are 16-byte multiples whose word pitch shifts successive rows
// across banks (88 bf16 = 44 words, 84 f32 = 84 words). MAXB boxes of 8 rows per stage:
// FP32 stages hold 64 rows, so three CTAs fit an SM (80-row FP32 stages allowed two, and
// the three-slice launch ran 18 % slower); taller footprints use the global-load path.
template <> struct StageGeom<__nv_bfloat16> { static constexpr int W = 88, ALIGN = 8, STAGES = 4, MAXB = 10; };
template <> struct StageGeom<__half> { static constexpr int W = 88, ALIGN = 8, STAGES = 4, MAXB = 10; };
template <> struct StageGeom<float> { static constexpr int W = 84, ALIGN = 4, STAGES = 3, MAXB = 8; };

enum : int { MODE_STAGED = 0, MODE_GLOBAL = 1, MODE_SKIP = 2 };

// What the consumer warps read per (tile, view): the local affine maps of the projective
// numerators u, v and denominator w, (value at the tile origin, d/di, d/dj), in stage-local
// coordinates, packed into three 16-byte words:
//   a = (u0, u_i, u_j, v0), b = (v_i, v_j, w0, w_i), c = (w_j, qscale, max tap offset, mode)
struct __align__(16) ViewRec {
    float4 a, b, c;
};
// The producer's copy adds the TMA box origin and count.
struct __align__(16) ViewMeta {
    ViewRec rec;
    int x0, r0, nbox, mode;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` polls and reports it (never spins forever).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (status) atomicExch(status, MR_ERR_TIMEOUT);
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ unsigned short lds_u16(uint32_t addr) {
    unsigned short u;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(u) : "r"(addr));
    return u;
}
// a - c, rounded to nearest, for a 16-bit value a (raw BF16 / FP16 bits) and an FP32 c
template <typename T>
__device__ __forceinline__ float sub16_f32(unsigned short a, float c) {
    float d;
    if constexpr (std::is_same<T, __nv_bfloat16>::value)
        asm("sub.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(a), "f"(c));
    else
        asm("sub.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(a), "f"(c));
    return d;
}

template <typename T>
__device__ __forceinline__ float lds_elem(uint32_t addr);
template <>
__device__ __forceinline__ float lds_elem<float>(uint32_t addr) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}
template <>
__device__ __forceinline__ float lds_elem<__nv_bfloat16>(uint32_t addr) {
    unsigned short u;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(u) : "r"(addr));
    return __uint_as_float(static_cast<uint32_t>(u) << 16);
}
template <>
__device__ __forceinline__ float lds_elem<__half>(uint32_t addr) {
    unsigned short u;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(u) : "r"(addr));
    return __half2float(__ushort_as_half(u));
}

// Global-memory bilinear (fallback for footprints larger than a stage).
template <typename T>
__device__ __forceinline__ float bilerp_global(const T* __restrict__ q, int R, int C, int pitch,
                                               float row, float col) {
    row = fminf(fmaxf(row, -2.f), (float)R + 1.f);
    col = fminf(fmaxf(col, -2.f), (float)C + 1.f);
    const float r0f = floorf(row), c0f = floorf(col);
    const float fr = row - r0f, fc = col - c0f;
    const int r0 = (int)r0f, c0 = (int)c0f;
    const bool rin0 = (unsigned)r0 < (unsigned)R, rin1 = (unsigned)(r0 + 1) < (unsigned)R;
    const bool cin0 = (unsigned)c0 < (unsigned)C, cin1 = (unsigned)(c0 + 1) < (unsigned)C;
    const T* p = q + (ptrdiff_t)r0 * pitch + c0;
    const float q00 = (rin0 && cin0) ? ld_elem(p) : 0.f;
    const float q01 = (rin0 && cin1) ? ld_elem(p + 1) : 0.f;
    const float q10 = (rin1 && cin0) ? ld_elem(p + pitch) : 0.f;
    const float q11 = (rin1 && cin1) ? ld_elem(p + pitch + 1) : 0.f;
    const float a = fmaf(fc, q01 - q00, q00);
    const float b = fmaf(fc, q11 - q10, q10);
    return fmaf(fr, b - a, a);
}

__device__ __forceinline__ bool in_box_fp64_t(const mr_grid& g, int i, int j) {
    const double aj = __dmul_rn((double)j - g.mask_half, g.mask_delta);
    const double ai = __dmul_rn((double)i - g.mask_half, g.mask_delta);
    bool ok = true;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const double p = __dadd_rn(__dadd_rn(g.mask_c[e], __dmul_rn(aj, g.mask_ej[e])),
                                   __dmul_rn(ai, g.mask_ei[e]));
        ok = ok && (fabs(p) <= g.box[e]);
    }
    return ok;
}

// Per-view footprint + local affine coefficients of one tile (computed by one lane of
// the producer warp).
template <int KIND, typename T>
__device__ __forceinline__ ViewMeta view_meta(const mr_view& V, const mr_grid& g, float ox, float oy,
                                              float oz, int di_max, int dj_max, int R, int C) {
    constexpr int W = StageGeom<T>::W;
    float pu[4], pv[4];
    view_map(V, g, R, C, pu, pv);
    auto aff = [&](const float* m) {
        return make_float3(fmaf(m[0], ox, fmaf(m[1], oy, fmaf(m[2], oz, m[3]))),
                           fmaf(m[0], g.step_i[0], fmaf(m[1], g.step_i[1], m[2] * g.step_i[2])),
                           fmaf(m[0], g.step_j[0], fmaf(m[1], g.step_j[1], m[2] * g.step_j[2])));
    };
    float3 au = aff(pu), av = aff(pv), aw = aff(V.pw);
    if (KIND == MR_CONE && V.qscale != 1.f) {
        // col = nu/nw and row = nv/nw are scale free, 1/nw^2 picks up qscale
        const float k = rsqrtf(V.qscale);
        au = make_float3(au.x * k, au.y * k, au.z * k);
        av = make_float3(av.x * k, av.y * k, av.z * k);
        aw = make_float3(aw.x * k, aw.y * k, aw.z * k);
    }
    float cmin = 3e38f, cmax = -3e38f, rmin = 3e38f, rmax = -3e38f;
    bool behind = false;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float di = (c & 1) ? (float)di_max : 0.f;
        const float dj = (c & 2) ? (float)dj_max : 0.f;
        const float w = fmaf(di, aw.y, fmaf(dj, aw.z, aw.x));
        float cc = fmaf(di, au.y, fmaf(dj, au.z, au.x));
        float rr = fmaf(di, av.y, fmaf(dj, av.z, av.x));
        if (KIND == MR_CONE) {
            behind |= !(w > 1e-3f);
            const float inv = 1.f / w;
            cc *= inv;
            rr *= inv;
        }
        cmin = fminf(cmin, cc); cmax = fmaxf(cmax, cc);
        rmin = fminf(rmin, rr); rmax = fmaxf(rmax, rr);
    }
    ViewMeta m;
    int mode = MODE_GLOBAL, x0 = 0, r0 = 0, nbox = 0;
    if (!behind && cmax == cmax && rmax == rmax && cmin == cmin && rmin == rmin) {
        if (cmax < -2.f || cmin > (float)C + 1.f || rmax < -2.f || rmin > (float)R + 1.f) {
            mode = MODE_SKIP;
        } else if (cmax - cmin < (float)(W - StageGeom<T>::ALIGN - 4) &&
                   rmax - rmin < (float)(ST_BOX_H * StageGeom<T>::MAXB - 4)) {
            x0 = ((int)floorf(cmin) - 1) & ~(StageGeom<T>::ALIGN - 1);
            r0 = (int)floorf(rmin) - 1;
            const int rows = (int)floorf(rmax) + 3 - r0;
            nbox = (rows + ST_BOX_H - 1) / ST_BOX_H;
            if ((int)floorf(cmax) + 3 - x0 <= W && nbox <= StageGeom<T>::MAXB) mode = MODE_STAGED;
        }
    }
    float3 cu = au, cv = av;
    if (mode == MODE_STAGED) {
        const float fx0 = (float)x0, fr0 = (float)r0;
        cu = make_float3(fmaf(-fx0, aw.x, au.x), fmaf(-fx0, aw.y, au.y), fmaf(-fx0, aw.z, au.z));
        cv = make_float3(fmaf(-fr0, aw.x, av.x), fmaf(-fr0, aw.y, av.y), fmaf(-fr0, aw.z, av.z));
    }
    // largest byte offset of a tap pair's left tap inside the staged boxes
    constexpr int ESZ = (int)sizeof(T);
    const uint32_t maxoff = mode == MODE_STAGED ? (uint32_t)(nbox * W * ST_BOX_H * ESZ - (W + 1) * ESZ - ESZ) : 0u;
    m.rec.a = make_float4(cu.x, cu.y, cu.z, cv.x);
    m.rec.b = make_float4(cv.y, cv.z, aw.x, aw.y);
    m.rec.c = make_float4(aw.z, V.qscale, __uint_as_float(maxoff), __int_as_float(mode));
    m.x0 = x0; m.r0 = r0; m.nbox = nbox; m.mode = mode;
    return m;
}

// Warp-specialised: warps 0..7 consume (256 threads x 4 samples = one 32x32 tile), warp 8
// produces. Stage s carries the TMA data and its ViewMeta; full[s] (1 arrival + TMA bytes)
// and empty[s] (one arrival per consumer warp) hand it back and forth. No CTA-wide barrier
// in the view loop, so consumer warps may run up to S views apart.
// A thread-block cluster of ST_CLUSTER CTAs shares one tile: CTA rank r back-projects the
// r-th quarter of the views and rank 0 sums the partials from the others' shared memory
// (DSMEM) in rank order - deterministic, no atomics, no scratch - and writes the tile.
// Three CTAs fit an SM (shared memory); the launch bound says so, or ptxas aims at four and
// spills the FP32 variant to fit its registers.
template <int KIND, typename T>
__global__ void __launch_bounds__(ST_THREADS, 3)
bp_staged_kernel(const __grid_constant__ CUtensorMap tmap, const T* __restrict__ ring, int R, int C,
                 int pitch, long long slot_stride, int n_slots, const mr_view* __restrict__ views,
                 const mr_grid* __restrict__ grids, const mr_tile* __restrict__ tiles,
                 float* __restrict__ out, int* status, const int64_t* __restrict__ n_tiles_dev,
                 unsigned int* __restrict__ counter, long long tile_cap) {
    constexpr int W = StageGeom<T>::W;
    constexpr int S = StageGeom<T>::STAGES;
    constexpr int ESZ = (int)sizeof(T);
    constexpr int STAGE_BYTES = W * ST_BOX_H * StageGeom<T>::MAXB * ESZ;
    constexpr int BOX_BYTES = W * ST_BOX_H * ESZ;
    // every TMA destination (stage start + b * BOX_BYTES) must be 128-byte aligned
    static_assert(BOX_BYTES % 128 == 0 && STAGE_BYTES % 128 == 0, "TMA box / stage not 128-byte aligned");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations must be 128-byte aligned: round the dynamic buffer up (the host
    // allocates 128 spare bytes), whatever static shared memory precedes it.
    unsigned char* stages = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
    ViewRec* meta_ring = reinterpret_cast<ViewRec*>(stages + S * STAGE_BYTES);     // S
    ViewMeta* meta_new = reinterpret_cast<ViewMeta*>(meta_ring + S);                // 32
    uint64_t* full = reinterpret_cast<uint64_t*>(meta_new + 32);                    // S
    uint64_t* empty = full + S;                                                      // S
    float4* partial = reinterpret_cast<float4*>(empty + S);                          // 256 (cluster sum)
    __shared__ mr_grid s_g;

    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = warp == ST_CONSUMERS;
    __shared__ unsigned int s_next;
    if (tid < S) {
        mbar_init(&full[tid], 1);
        mbar_init(&empty[tid], ST_CONSUMERS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    uint32_t used = 0;              // views this CTA has put through the stage ring so far

    // One tile per cluster (counter == nullptr), or persistent: clusters pull tile indices
    // from the device work counter until it passes *n_tiles_dev.
    for (int iter = 0;; ++iter) {
        long long tile_idx;
        if (counter) {
            // rank 0 pushes the tile index into every CTA's own shared memory before the
            // barrier; after it each CTA reads only its local copy, so no CTA touches a
            // peer's shared memory once the cluster may start exiting (the final break)
            if (crank == 0 && tid == 0) {
                const unsigned int nx = atomicAdd(counter, 1u);
                for (int r = 0; r < csize; ++r) *cluster.map_shared_rank(&s_next, r) = nx;
            }
            cluster.sync();
            tile_idx = (long long)s_next;
            // the device count is clamped to the capacity of the tile buffer
            if (tile_idx >= min((long long)*n_tiles_dev, tile_cap)) break;
        } else {
            if (iter > 0) break;
            tile_idx = (long long)(blockIdx.x / csize);
        }
        const mr_tile t = tiles[tile_idx];
        __syncthreads();                    // previous tile's readers of s_g are done
        if (tid < (int)(sizeof(mr_grid) / 4))
            reinterpret_cast<int*>(&s_g)[tid] = reinterpret_cast<const int*>(grids + t.grid)[tid];
        __syncthreads();
        const mr_grid& g = s_g;
        // this CTA's share of the views: [v_begin, v_end)
        int first, count;                   // the grid's slots [first, first + count)
        grid_view_range(g.view_begin, g.n_views, n_slots, &first, &count);
        const int v_begin = first + (int)(((long long)count * crank) / csize);
        const int v_end = first + (int)(((long long)count * (crank + 1)) / csize);
        const int nv = v_end - v_begin;

        const float ox = g.origin[0] + t.i0 * g.step_i[0] + t.j0 * g.step_j[0] + t.k * g.step_k[0];
        const float oy = g.origin[1] + t.i0 * g.step_i[1] + t.j0 * g.step_j[1] + t.k * g.step_k[1];
        const float oz = g.origin[2] + t.i0 * g.step_i[2] + t.j0 * g.step_j[2] + t.k * g.step_k[2];
        // warp w covers columns 16 (w & 1) .. + 15 and rows 8 (w >> 1) .. + 7 of the tile; its
        // p-th sample step is a 16 x 2 patch (rows ty + 2p). The patch shape keeps the 32
        // lanes' bilinear taps on distinct shared-memory banks for most plane orientations
        // (1.10 wavefronts per 16-bit tap load on the bench slices, 1.35 for 8 x 4 patches)
        // and makes each half-warp's output a 64-byte row segment.
        const int tx = ((warp & 1) << 4) | (lane & 15);
        const int ty = ((warp >> 1) << 3) | (lane >> 4);
        bool inside[ST_PPT];
        bool any = false;
#pragma unroll
        for (int p = 0; p < ST_PPT; ++p) {
            const int i = t.i0 + ty + ST_DI * p, j = t.j0 + tx;
            bool ok = !producer && i < g.n_i && j < g.n_j;
            if (ok && (g.flags & MR_GRID_MASK_BOX)) ok = in_box_fp64_t(g, i, j);
            inside[p] = ok;
            any |= ok;
        }
        const bool tile_live = __syncthreads_or(any) != 0;
        // warp-uniform: an 8x4 sample patch wholly outside the box is not computed
        bool wlive[ST_PPT];
#pragma unroll
        for (int p = 0; p < ST_PPT; ++p) wlive[p] = __any_sync(0xffffffffu, inside[p]);

        if (producer && tile_live) {
            const int di_max = min(ST_TI, g.n_i - t.i0) - 1;
            const int dj_max = min(ST_TJ, g.n_j - t.j0) - 1;
            for (int vb = 0; vb < nv; vb += 32) {
                const int cnt = min(32, nv - vb);
                __syncwarp();
                if (lane < cnt)
                    meta_new[lane] = view_meta<KIND, T>(views[v_begin + vb + lane], g, ox, oy, oz, di_max,
                                                        dj_max, R, C);
                __syncwarp();
                // lane 0 frees and arms the stage, then lane b issues the copy of box b: the
                // boxes of a view go out in one warp instruction instead of one after another
                for (int l = 0; l < cnt; ++l) {
                    const uint32_t ua = used + (uint32_t)(vb + l);          // absolute stage use
                    const int s = (int)(ua % S);
                    const uint32_t u = ua / S;
                    const int mode = meta_new[l].mode, nbox = meta_new[l].nbox;
                    if (lane == 0) {
                        if (u > 0) mbar_wait(&empty[s], (u - 1) & 1u, status);
                        meta_ring[s] = meta_new[l].rec;
                        if (mode == MODE_STAGED) mbar_arrive_tx(&full[s], (uint32_t)(nbox * BOX_BYTES));
                        else mbar_arrive(&full[s]);
                    }
                    __syncwarp();                   // the stage is free and armed for every lane
                    if (mode == MODE_STAGED && lane < nbox)
                        tma_load_3d(stages + s * STAGE_BYTES + lane * BOX_BYTES, &tmap, meta_new[l].x0,
                                    meta_new[l].r0 + lane * ST_BOX_H, v_begin + vb + l, &full[s]);
                }
            }
        }

        // sample p sits in pair p / 2, lane p % 2 (pairs of rows i and i + ST_DI)
        float2 acc2[ST_PPT / 2];
        float2 fi2[ST_PPT / 2];
#pragma unroll
        for (int h = 0; h < ST_PPT / 2; ++h) {
            acc2[h] = make_float2(0.f, 0.f);
            fi2[h] = make_float2((float)(ty + 2 * ST_DI * h), (float)(ty + 2 * ST_DI * h + ST_DI));
        }
        if (!producer && tile_live) {
            const float fj = (float)tx;
            int s = (int)(used % S);                    // stage of view 0 of this tile
            uint32_t phase = (used / S) & 1u;           // and the parity of its fill
            for (int v = 0; v < nv; ++v) {
                mbar_wait(&full[s], phase, status);
                const ViewRec m = meta_ring[s];
                const int mode = __float_as_int(m.c.w);
                const float bu = fmaf(fj, m.a.z, m.a.x);
                const float bv = fmaf(fj, m.b.y, m.a.w);
                const float bw = fmaf(fj, m.c.x, m.b.z);
                if (mode == MODE_STAGED) {
                    const uint32_t base = smem_u32(stages + s * STAGE_BYTES);
                    const uint32_t maxoff = __float_as_uint(m.c.z);
                    // byte offset = (bits_r - MAGIC_BITS) * W*ESZ + (bits_c - MAGIC_BITS) * ESZ
                    const uint32_t kofs = (uint32_t)MAGIC_BITS * (uint32_t)(W * ESZ + ESZ);
                    // Two samples (rows i and i + 2) per packed f32x2 instruction: every
                    // component is the scalar FMA / add / multiply it replaces, so the result
                    // is the same bit for bit; only the issue slots halve.
                    const float2 cuy = make_float2(m.a.y, m.a.y), cvy = make_float2(m.b.x, m.b.x);
                    const float2 cwy = make_float2(m.b.w, m.b.w);
                    const float2 bu2 = make_float2(bu, bu), bv2 = make_float2(bv, bv), bw2 = make_float2(bw, bw);
#pragma unroll
                    for (int h = 0; h < ST_PPT / 2; ++h) {
                        if (!(wlive[2 * h] | wlive[2 * h + 1])) continue;
                        const float2 nu = __ffma2_rn(fi2[h], cuy, bu2);
                        const float2 nv2 = __ffma2_rn(fi2[h], cvy, bv2);
                        float2 r = make_float2(1.f, 1.f), yc, yr, fc, fr;
                        if (KIND == MR_CONE) {
                            const float2 w = __ffma2_rn(fi2[h], cwy, bw2);
                            r = make_float2(rcp_approx(w.x), rcp_approx(w.y));
                            yc = __ffma2_rd(nu, r, kMagic2);
                            yr = __ffma2_rd(nv2, r, kMagic2);
                            // MAGIC - y is exact; fma(y, -1, MAGIC) is that subtraction
                            fc = __ffma2_rn(nu, r, __ffma2_rn(yc, kNeg2, kMagic2));
                            fr = __ffma2_rn(nv2, r, __ffma2_rn(yr, kNeg2, kMagic2));
                        } else {
                            yc = __fadd2_rd(nu, kMagic2);
                            yr = __fadd2_rd(nv2, kMagic2);
                            fc = __fadd2_rn(nu, __ffma2_rn(yc, kNeg2, kMagic2));
                            fr = __fadd2_rn(nv2, __ffma2_rn(yr, kNeg2, kMagic2));
                        }
                        uint32_t a[2];
                        a[0] = base + min((uint32_t)__float_as_int(yr.x) * (uint32_t)(W * ESZ) +
                                              (uint32_t)__float_as_int(yc.x) * (uint32_t)ESZ - kofs, maxoff);
                        a[1] = base + min((uint32_t)__float_as_int(yr.y) * (uint32_t)(W * ESZ) +
                                              (uint32_t)__float_as_int(yc.y) * (uint32_t)ESZ - kofs, maxoff);
                        float2 q00, q10, d0, d1;
                        if constexpr (sizeof(T) == 2) {
                            // the right taps stay 16-bit: one mixed-precision subtraction each
                            // (16-bit values widen exactly, so it is the FP32 difference)
                            q00 = make_float2(lds_elem<T>(a[0]), lds_elem<T>(a[1]));
                            q10 = make_float2(lds_elem<T>(a[0] + W * ESZ), lds_elem<T>(a[1] + W * ESZ));
                            d0 = make_float2(sub16_f32<T>(lds_u16(a[0] + ESZ), q00.x),
                                             sub16_f32<T>(lds_u16(a[1] + ESZ), q00.y));
                            d1 = make_float2(sub16_f32<T>(lds_u16(a[0] + W * ESZ + ESZ), q10.x),
                                             sub16_f32<T>(lds_u16(a[1] + W * ESZ + ESZ), q10.y));
                        } else {
                            q00 = make_float2(lds_elem<T>(a[0]), lds_elem<T>(a[1]));
                            q10 = make_float2(lds_elem<T>(a[0] + W * ESZ), lds_elem<T>(a[1] + W * ESZ));
                            const float2 q01 = make_float2(lds_elem<T>(a[0] + ESZ), lds_elem<T>(a[1] + ESZ));
                            const float2 q11 = make_float2(lds_elem<T>(a[0] + W * ESZ + ESZ),
                                                           lds_elem<T>(a[1] + W * ESZ + ESZ));
                            d0 = __ffma2_rn(q00, kNeg2, q01);          // q01 - q00
                            d1 = __ffma2_rn(q10, kNeg2, q11);          // q11 - q10
                        }
                        const float2 ta = __ffma2_rn(fc, d0, q00);
                        const float2 tb = __ffma2_rn(fc, d1, q10);
                        const float2 val = __ffma2_rn(fr, __ffma2_rn(ta, kNeg2, tb), ta);
                        const float2 wgt = KIND == MR_CONE ? __fmul2_rn(r, r) : make_float2(m.c.y, m.c.y);
                        acc2[h] = __ffma2_rn(wgt, val, acc2[h]);
                    }
                } else if (mode == MODE_GLOBAL) {
                    const T* q = ring + (long long)(v_begin + v) * slot_stride;
#pragma unroll
                    for (int p = 0; p < ST_PPT; ++p) {
                        if (!wlive[p]) continue;
                        const float fi = (float)(ty + ST_DI * p);
                        const float nu = fmaf(fi, m.a.y, bu);
                        const float nvv = fmaf(fi, m.b.x, bv);
                        float& ap = (p & 1) ? acc2[p >> 1].y : acc2[p >> 1].x;
                        if (KIND == MR_CONE) {
                            const float r = rcp_approx(fmaf(fi, m.b.w, bw));
                            ap = fmaf(r * r, bilerp_global(q, R, C, pitch, nvv * r, nu * r), ap);
                        } else {
                            ap = fmaf(m.c.y, bilerp_global(q, R, C, pitch, nvv, nu), ap);
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);      // this warp is done with stage s
                if (++s == S) {
                    s = 0;
                    phase ^= 1u;
                }
            }
        }
        if (tile_live) used += (uint32_t)nv;

        // ---- cluster reduction of the view-quarter partial sums (rank order), rank 0 writes
        float acc[ST_PPT] = {acc2[0].x, acc2[0].y, acc2[1].x, acc2[1].y};
        if (csize > 1) {
            if (!producer) partial[tid] = make_float4(acc[0], acc[1], acc[2], acc[3]);
            cluster.sync();
            if (crank == 0 && !producer) {
                for (int r = 1; r < csize; ++r) {
                    const float4 o = cluster.map_shared_rank(partial, r)[tid];
                    acc[0] += o.x; acc[1] += o.y; acc[2] += o.z; acc[3] += o.w;
                }
            }
        }
        if (crank == 0 && !producer) {
#pragma unroll
            for (int p = 0; p < ST_PPT; ++p) {
                const int i = t.i0 + ty + ST_DI * p, j = t.j0 + tx;
                if (i < g.n_i && j < g.n_j) {
                    const long long o = g.out_offset + (long long)i * g.out_stride_i +
                                        (long long)j * g.out_stride_j + (long long)t.k * g.out_stride_k;
                    const float val = inside[p] ? acc[p] * g.scale : 0.f;
                    out[o] = g.accumulate ? out[o] + val : val;
                }
            }
        }
        if (csize > 1) cluster.sync();      // keep every partial alive until rank 0 has read it
    }
}

// ---------------------------------------------------------------- host side
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <typename T>
static int make_ring_map(const mr_ring* ring, CUtensorMap* map) {
    auto fn = encode_fn();
    if (!fn) return MR_ERR_CUDA;
    const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : (std::is_same<T, __half>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                     : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16);
    const cuuint64_t dims[3] = {(cuuint64_t)ring->cols, (cuuint64_t)ring->rows, (cuuint64_t)ring->n_slots};
    const cuuint64_t strides[2] = {(cuuint64_t)ring->col_pitch * sizeof(T),
                                   (cuuint64_t)ring->slot_stride * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)StageGeom<T>::W, (cuuint32_t)ST_BOX_H, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dt, 3, ring->data, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MR_OK : MR_ERR_INVALID;
}

template <int KIND, typename T>
static int launch_staged(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                         const mr_tile* tiles, int64_t n_tiles, float* out, int* status, cudaStream_t st,
                         const int64_t* n_tiles_dev = nullptr, unsigned int* counter = nullptr) {
    CUtensorMap map;
    int rc = make_ring_map<T>(ring, &map);
    if (rc != MR_OK) return rc;
    constexpr int S = StageGeom<T>::STAGES;
    const size_t smem = (size_t)S * StageGeom<T>::W * ST_BOX_H * StageGeom<T>::MAXB * sizeof(T) +
                        S * sizeof(ViewRec) + 32 * sizeof(ViewMeta) + 2 * S * sizeof(uint64_t) +
                        ST_CONSUMERS * 32 * sizeof(float4) + 128;
    auto kern = bp_staged_kernel<KIND, T>;
    MR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(ST_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ST_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (counter) {
        // persistent: as many clusters as fit at once, pulling tiles from the counter
        int clusters = 0;
        cfg.gridDim = dim3(ST_CLUSTER);
        MR_CUDA_TRY(cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg));
        if (clusters < 1) clusters = 1;
        if ((int64_t)clusters > n_tiles) clusters = (int)(n_tiles > 0 ? n_tiles : 1);
        MR_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st));
        cfg.gridDim = dim3((unsigned)(clusters * ST_CLUSTER));
        MR_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, map, static_cast<const T*>(ring->data), ring->rows, ring->cols,
                                       ring->col_pitch, (long long)ring->slot_stride, (int)ring->n_slots, views,
                                       grids, tiles, out, status, n_tiles_dev, counter, (long long)n_tiles));
    } else {
        const int64_t max_chunk = 2147483647LL / ST_CLUSTER;
        for (int64_t t0 = 0; t0 < n_tiles; t0 += max_chunk) {
            const int64_t n = (n_tiles - t0) < max_chunk ? (n_tiles - t0) : max_chunk;
            cfg.gridDim = dim3((unsigned)(n * ST_CLUSTER));
            MR_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, map, static_cast<const T*>(ring->data), ring->rows,
                                           ring->cols, ring->col_pitch, (long long)ring->slot_stride,
                                           (int)ring->n_slots, views, grids, tiles + t0, out, status,
                                           (const int64_t*)nullptr, (unsigned int*)nullptr, (long long)n));
        }
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

static int check_staged_ring(const mr_ring* ring) {
    if (!ring || !ring->data) return MR_ERR_INVALID;
    if (ring->rows <= 0 || ring->cols <= 0 || ring->col_pitch < ring->cols || ring->n_slots <= 0)
        return MR_ERR_INVALID;
    if (ring->slot_stride < (int64_t)ring->rows * ring->col_pitch) return MR_ERR_INVALID;
    if (ring->kind != MR_CONE && ring->kind != MR_PARALLEL) return MR_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(ring->data) & 15) != 0) return MR_ERR_INVALID;
    const int esz = ring->dtype == MR_F32 ? 4 : 2;
    if (ring->dtype != MR_F32 && ring->dtype != MR_BF16 && ring->dtype != MR_F16) return MR_ERR_INVALID;
    if ((ring->col_pitch * esz) % 16 || (ring->slot_stride * esz) % 16) return MR_ERR_INVALID;
    return MR_OK;
}

template <typename... Args>
static int dispatch_staged(const mr_ring* ring, Args... args) {
    const bool cone = ring->kind == MR_CONE;
    switch (ring->dtype) {
        case MR_F32:
            return cone ? launch_staged<MR_CONE, float>(ring, args...) : launch_staged<MR_PARALLEL, float>(ring, args...);
        case MR_BF16:
            return cone ? launch_staged<MR_CONE, __nv_bfloat16>(ring, args...)
                        : launch_staged<MR_PARALLEL, __nv_bfloat16>(ring, args...);
        default:
            return cone ? launch_staged<MR_CONE, __half>(ring, args...) : launch_staged<MR_PARALLEL, __half>(ring, args...);
    }
}

}  // namespace mr

extern "C" int mr_backproject_staged(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                                     const mr_tile* tiles, int64_t n_tiles, float* out, int32_t* status,
                                     void* stream) {
    int rc = mr::check_staged_ring(ring);
    if (rc != MR_OK) return rc;
    if (!views || !grids || !out || n_tiles < 0 || (n_tiles > 0 && !tiles)) return MR_ERR_INVALID;
    if (n_tiles == 0) return MR_OK;
    return mr::dispatch_staged(ring, views, grids, tiles, n_tiles, out, status, static_cast<cudaStream_t>(stream),
                               (const int64_t*)nullptr, (unsigned int*)nullptr);
}

extern "C" int mr_backproject_persistent(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                                         const mr_tile* tiles, const int64_t* n_tiles_dev, int64_t max_tiles,
                                         uint32_t* counter_dev, float* out, int32_t* status, void* stream) {
    int rc = mr::check_staged_ring(ring);
    if (rc != MR_OK) return rc;
    if (!views || !grids || !tiles || !n_tiles_dev || !counter_dev || !out || max_tiles < 1) return MR_ERR_INVALID;
    // the 32-bit work counter must not wrap while the last clusters overshoot the count
    if (max_tiles > (int64_t(1) << 31)) return MR_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(counter_dev) & 3) != 0) return MR_ERR_INVALID;
    return mr::dispatch_staged(ring, views, grids, tiles, max_tiles, out, status, static_cast<cudaStream_t>(stream),
                               n_tiles_dev, reinterpret_cast<unsigned int*>(counter_dev));
}

// ---------------------------------------------------------------- no-allocation variant
// The persistent launch needs one 32-bit work counter in device memory. Callers that
// cannot allocate device memory get it from this file-scope array instead; every GPU that
// loads the library holds it until the process exits, and every call shares it.
static __device__ __align__(256) unsigned int g_noalloc_scratch[MR_NOALLOC_SCRATCH_BYTES / 4];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned int* g_noalloc_addr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once per device.
// In host code the array's name is only a host-side stand-in, never a device address.
int noalloc_counter(cudaStream_t stream, unsigned int** counter) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return MR_ERR_CUDA;
    if (dev >= kNoallocMaxDevices) return MR_ERR_UNSUPPORTED;
    if (stream) {
        int sdev = -1;
        if (cudaStreamGetDevice(stream, &sdev) != cudaSuccess) return MR_ERR_CUDA;
        if (sdev != dev) return MR_ERR_INVALID;      // the stream's device must be current
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        // the symbol lookup may load device code, which a capture in progress forbids
        if (stream) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
                cudaGetLastError();
                return MR_ERR_CUDA;
            }
            if (cs != cudaStreamCaptureStatusNone) return MR_ERR_CAPTURE;
        }
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return MR_ERR_CUDA;
        }
        g_noalloc_addr[dev] = static_cast<unsigned int*>(p);
    }
    *counter = g_noalloc_addr[dev];
    return MR_OK;
}
}  // namespace

extern "C" int mr_backproject_persistent_noalloc(const mr_ring* ring, const mr_view* views,
                                                 const mr_grid* grids, const mr_tile* tiles,
                                                 const int64_t* n_tiles_dev, int64_t max_tiles, float* out,
                                                 int32_t* status, void* stream) {
    int rc = mr::check_staged_ring(ring);
    if (rc != MR_OK) return rc;
    if (!views || !grids || !tiles || !n_tiles_dev || !out || max_tiles < 1) return MR_ERR_INVALID;
    if (max_tiles > MR_NOALLOC_MAX_TILES) return MR_ERR_SCRATCH_LIMIT;
    unsigned int* counter = nullptr;
    rc = noalloc_counter(static_cast<cudaStream_t>(stream), &counter);
    if (rc != MR_OK) return rc;
    // the shared launch path zeroes the counter on `stream` before the kernel
    return mr::dispatch_staged(ring, views, grids, tiles, max_tiles, out, status, static_cast<cudaStream_t>(stream),
                               n_tiles_dev, counter);
}
