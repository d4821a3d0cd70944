// Voxel-driven back-projection over a device-resident filtered-projection ring.
//
// Reference semantics (minirecast recon.py):
//   bp_cone_numba   193-219: f(p) = scale * sum_k (SOD_k/L_k)^2 * bilerp(q_k, row_k(p), col_k(p))
//   bp_parallel_numba 175-191: the same with an affine projection and weight 1
//   _bil_nb         156-173: bilinear, every tap outside [0,R)x[0,C) contributes 0
//   reconstruct_points 405-424: COR shift D = d - shift*u  (folded here into the
//                    projective map: col += shift, row += shift * (u.v)/|v|^2)
//
// One CTA owns one tile of one grid (request); a launch may mix tiles of many grids
// of any size / zoom / orientation. Each thread keeps PPT samples in FP32 registers
// and walks all views of its grid. Per view, the CTA turns the view's 3x4 map into
// affine coefficients relative to the tile origin (staged in shared memory), so the
// per-sample cost is 3 FMA + 1 RCP + 3 MUL + bilinear.
#include "mr_common.cuh"

namespace mr {

constexpr int BP_TJ = 32;              // samples along j per tile (threadIdx.x)
constexpr int BP_TY = 8;               // threadIdx.y
constexpr int BP_PPT = 4;              // samples per thread along i
constexpr int BP_TI = BP_TY * BP_PPT;  // samples along i per tile
constexpr int BP_THREADS = BP_TJ * BP_TY;
constexpr int BP_PTS_PER_TILE = BP_THREADS * BP_PPT;
constexpr int BP_VCH = 128;            // views staged per shared-memory chunk

template <typename T>
__device__ __forceinline__ float bilerp(const T* __restrict__ q, int R, int C, int pitch,
                                        float row, float col) {
    // Clamp far-away coordinates (and NaN) into a range whose taps are all outside
    // the detector, so the integer conversion cannot overflow.
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

// Box mask of a plane sample in FP64 with the rounding order of minirecast
// slice_points / plane_points (recon.py:238-265): p = (c + a_j e_j) + a_i e_i,
// a_x = (x - (n-1)/2) * (size/n); kept when |p| <= box on every axis.
__device__ __forceinline__ bool in_box_fp64(const mr_grid& g, int i, int j) {
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

__device__ __forceinline__ float dot3(const float* a, float x, float y, float z) {
    return fmaf(a[0], x, fmaf(a[1], y, a[2] * z));
}

template <int KIND, typename T>
__global__ void __launch_bounds__(BP_THREADS)
bp_kernel(const T* __restrict__ ring_all, int R, int C, int pitch, long long slot_stride, int n_slots,
          const mr_view* __restrict__ views_all, const mr_grid* __restrict__ grids,
          const mr_tile* __restrict__ tiles, float* __restrict__ out) {
    __shared__ float4 s_u[BP_VCH], s_v[BP_VCH], s_w[BP_VCH];
    __shared__ float s_q[BP_VCH];
    __shared__ mr_grid s_g;

    const mr_tile t = tiles[blockIdx.x];
    const int tid = threadIdx.y * BP_TJ + threadIdx.x;
    // Each warp covers compact 8 (j) x 4 (i) sample patches, so the detector footprint
    // of one warp-wide gather is a small 2D patch whatever the plane orientation.
    const int warp = tid >> 5, lane = tid & 31;
    const int tx = ((warp & 3) << 3) | (lane & 7);            // j offset in the tile, 0..31
    const int ty = ((warp >> 2) << 4) | (lane >> 3);          // i offset of p = 0; +4 per p
    if (tid < (int)(sizeof(mr_grid) / 4))
        reinterpret_cast<int*>(&s_g)[tid] = reinterpret_cast<const int*>(grids + t.grid)[tid];
    __syncthreads();
    const mr_grid& g = s_g;
    const bool points = (g.flags & MR_GRID_POINTS) != 0;
    // the grid sums slots [first, first + nv)
    int first, nv;
    grid_view_range(g.view_begin, g.n_views, n_slots, &first, &nv);
    const mr_view* __restrict__ views = views_all + first;
    const T* __restrict__ ring = ring_all + (long long)first * slot_stride;

    float acc[BP_PPT];
#pragma unroll
    for (int p = 0; p < BP_PPT; ++p) acc[p] = 0.f;

    if (!points) {
        // ---------------- regular grid: affine coefficients per view ----------------
        const float ox = g.origin[0] + t.i0 * g.step_i[0] + t.j0 * g.step_j[0] + t.k * g.step_k[0];
        const float oy = g.origin[1] + t.i0 * g.step_i[1] + t.j0 * g.step_j[1] + t.k * g.step_k[1];
        const float oz = g.origin[2] + t.i0 * g.step_i[2] + t.j0 * g.step_j[2] + t.k * g.step_k[2];
        const float fj = (float)tx;
        bool inside[BP_PPT];
        bool any = false;
#pragma unroll
        for (int p = 0; p < BP_PPT; ++p) {
            const int i = t.i0 + ty + 4 * p, j = t.j0 + tx;
            bool ok = i < g.n_i && j < g.n_j;
            if (ok && (g.flags & MR_GRID_MASK_BOX)) ok = in_box_fp64(g, i, j);
            inside[p] = ok;
            any |= ok;
        }
        const bool tile_live = __syncthreads_or(any) != 0;
        if (tile_live) {
            for (int v0 = 0; v0 < nv; v0 += BP_VCH) {
                const int nch = min(BP_VCH, nv - v0);
                __syncthreads();
                if (tid < nch) {
                    const mr_view V = views[v0 + tid];
                    float pu[4], pv[4];
                    view_map(V, g, R, C, pu, pv);
                    s_u[tid] = make_float4(dot3(pu, ox, oy, oz) + pu[3],
                                           dot3(pu, g.step_i[0], g.step_i[1], g.step_i[2]),
                                           dot3(pu, g.step_j[0], g.step_j[1], g.step_j[2]), V.qscale);
                    s_v[tid] = make_float4(dot3(pv, ox, oy, oz) + pv[3],
                                           dot3(pv, g.step_i[0], g.step_i[1], g.step_i[2]),
                                           dot3(pv, g.step_j[0], g.step_j[1], g.step_j[2]), 0.f);
                    s_w[tid] = make_float4(dot3(V.pw, ox, oy, oz) + V.pw[3],
                                           dot3(V.pw, g.step_i[0], g.step_i[1], g.step_i[2]),
                                           dot3(V.pw, g.step_j[0], g.step_j[1], g.step_j[2]), 0.f);
                }
                __syncthreads();
#pragma unroll 2
                for (int vv = 0; vv < nch; ++vv) {
                    const float4 cu = s_u[vv], cv = s_v[vv];
                    const T* q = ring + (long long)(v0 + vv) * slot_stride;
                    const float bu = fmaf(fj, cu.z, cu.x);
                    const float bv = fmaf(fj, cv.z, cv.x);
                    if (KIND == MR_CONE) {
                        const float4 cw = s_w[vv];
                        const float bw = fmaf(fj, cw.z, cw.x);
#pragma unroll
                        for (int p = 0; p < BP_PPT; ++p) {
                            const float fi = (float)(ty + 4 * p);
                            const float nu = fmaf(fi, cu.y, bu);
                            const float nvv = fmaf(fi, cv.y, bv);
                            const float nw = fmaf(fi, cw.y, bw);
                            const float r = rcp_approx(nw);
                            const float val = bilerp(q, R, C, pitch, nvv * r, nu * r);
                            acc[p] = fmaf(r * r * cu.w, val, acc[p]);
                        }
                    } else {
#pragma unroll
                        for (int p = 0; p < BP_PPT; ++p) {
                            const float fi = (float)(ty + 4 * p);
                            const float val = bilerp(q, R, C, pitch, fmaf(fi, cv.y, bv), fmaf(fi, cu.y, bu));
                            acc[p] = fmaf(cu.w, val, acc[p]);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int p = 0; p < BP_PPT; ++p) {
            const int i = t.i0 + ty + 4 * p, j = t.j0 + tx;
            if (i < g.n_i && j < g.n_j) {
                const long long o = g.out_offset + (long long)i * g.out_stride_i +
                                    (long long)j * g.out_stride_j + (long long)t.k * g.out_stride_k;
                const float val = inside[p] ? acc[p] * g.scale : 0.f;
                out[o] = g.accumulate ? out[o] + val : val;
            }
        }
    } else {
        // ---------------- explicit point list: full 3x4 map per view ----------------
        float px[BP_PPT], py[BP_PPT], pz[BP_PPT];
        bool ok[BP_PPT];
#pragma unroll
        for (int p = 0; p < BP_PPT; ++p) {
            const int j = t.j0 + tid + BP_THREADS * p;
            ok[p] = j < g.n_j;
            const int jj = ok[p] ? j : 0;
            px[p] = ok[p] ? g.points[3 * jj + 0] : 0.f;
            py[p] = ok[p] ? g.points[3 * jj + 1] : 0.f;
            pz[p] = ok[p] ? g.points[3 * jj + 2] : 0.f;
        }
        for (int v0 = 0; v0 < nv; v0 += BP_VCH) {
            const int nch = min(BP_VCH, nv - v0);
            __syncthreads();
            if (tid < nch) {
                const mr_view V = views[v0 + tid];
                float pu[4], pv[4];
                view_map(V, g, R, C, pu, pv);
                const float4 u = make_float4(pu[0], pu[1], pu[2], pu[3]);
                const float4 vq = make_float4(pv[0], pv[1], pv[2], pv[3]);
                const float4 w = make_float4(V.pw[0], V.pw[1], V.pw[2], V.pw[3]);
                s_u[tid] = u;
                s_v[tid] = vq;
                s_w[tid] = w;
                s_q[tid] = V.qscale;
            }
            __syncthreads();
            for (int vv = 0; vv < nch; ++vv) {
                const float4 cu = s_u[vv], cv = s_v[vv], cw = s_w[vv];
                const float qs = s_q[vv];
                const T* q = ring + (long long)(v0 + vv) * slot_stride;
#pragma unroll
                for (int p = 0; p < BP_PPT; ++p) {
                    const float nu = fmaf(cu.x, px[p], fmaf(cu.y, py[p], fmaf(cu.z, pz[p], cu.w)));
                    const float nvv = fmaf(cv.x, px[p], fmaf(cv.y, py[p], fmaf(cv.z, pz[p], cv.w)));
                    if (KIND == MR_CONE) {
                        const float nw = fmaf(cw.x, px[p], fmaf(cw.y, py[p], fmaf(cw.z, pz[p], cw.w)));
                        const float r = rcp_approx(nw);
                        const float val = bilerp(q, R, C, pitch, nvv * r, nu * r);
                        acc[p] = fmaf(r * r * qs, val, acc[p]);
                    } else {
                        acc[p] = fmaf(qs, bilerp(q, R, C, pitch, nvv, nu), acc[p]);
                    }
                }
            }
        }
#pragma unroll
        for (int p = 0; p < BP_PPT; ++p) {
            const int j = t.j0 + tid + BP_THREADS * p;
            if (ok[p]) {
                float* o = out + g.out_offset + (long long)j * g.out_stride_j;
                *o = g.accumulate ? *o + acc[p] * g.scale : acc[p] * g.scale;
            }
        }
    }
}

template <int KIND, typename T>
static int launch_bp(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                     const mr_tile* tiles, int64_t n_tiles, float* out, cudaStream_t st) {
    const dim3 block(BP_TJ, BP_TY);
    // gridDim.x limit is 2^31-1; tiles beyond that are launched in chunks.
    const int64_t max_chunk = 2147483647LL;
    for (int64_t t0 = 0; t0 < n_tiles; t0 += max_chunk) {
        const int64_t n = (n_tiles - t0) < max_chunk ? (n_tiles - t0) : max_chunk;
        bp_kernel<KIND, T><<<(unsigned)n, block, 0, st>>>(
            static_cast<const T*>(ring->data), ring->rows, ring->cols, ring->col_pitch,
            (long long)ring->slot_stride, (int)ring->n_slots, views, grids, tiles + t0, out);
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

}  // namespace mr

extern "C" void mr_bp_tile_shape(int32_t* tile_i, int32_t* tile_j) {
    if (tile_i) *tile_i = mr::BP_TI;
    if (tile_j) *tile_j = mr::BP_TJ;
}

extern "C" int mr_plan_tiles(const mr_grid* grids, int32_t n_grids, mr_tile* tiles,
                             int64_t capacity, int64_t* n_tiles) {
    if (!grids || n_grids < 0 || !n_tiles || capacity < 0 || (capacity > 0 && !tiles))
        return MR_ERR_INVALID;
    int64_t n = 0;
    for (int32_t g = 0; g < n_grids; ++g) {
        const mr_grid& G = grids[g];
        if (G.n_i < 0 || G.n_j < 0 || G.n_k < 0) return MR_ERR_INVALID;
        if (G.flags & MR_GRID_POINTS) {
            for (int32_t j0 = 0; j0 < G.n_j; j0 += mr::BP_PTS_PER_TILE) {
                if (n < capacity) tiles[n] = mr_tile{g, 0, j0, 0};
                ++n;
            }
        } else {
            for (int32_t k = 0; k < G.n_k; ++k)
                for (int32_t i0 = 0; i0 < G.n_i; i0 += mr::BP_TI)
                    for (int32_t j0 = 0; j0 < G.n_j; j0 += mr::BP_TJ) {
                        if (n < capacity) tiles[n] = mr_tile{g, i0, j0, k};
                        ++n;
                    }
        }
    }
    *n_tiles = n;
    return MR_OK;
}

extern "C" int mr_backproject(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                              const mr_tile* tiles, int64_t n_tiles, float* out, void* stream) {
    if (!ring || !ring->data || !views || !grids || !out || n_tiles < 0) return MR_ERR_INVALID;
    if (n_tiles > 0 && !tiles) return MR_ERR_INVALID;
    if (ring->rows <= 0 || ring->cols <= 0 || ring->col_pitch < ring->cols) return MR_ERR_INVALID;
    if (ring->slot_stride < (int64_t)ring->rows * ring->col_pitch) return MR_ERR_INVALID;
    if (ring->kind != MR_CONE && ring->kind != MR_PARALLEL) return MR_ERR_INVALID;
    if (n_tiles == 0) return MR_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool cone = ring->kind == MR_CONE;
    switch (ring->dtype) {
        case MR_F32:
            return cone ? mr::launch_bp<MR_CONE, float>(ring, views, grids, tiles, n_tiles, out, st)
                        : mr::launch_bp<MR_PARALLEL, float>(ring, views, grids, tiles, n_tiles, out, st);
        case MR_BF16:
            return cone ? mr::launch_bp<MR_CONE, __nv_bfloat16>(ring, views, grids, tiles, n_tiles, out, st)
                        : mr::launch_bp<MR_PARALLEL, __nv_bfloat16>(ring, views, grids, tiles, n_tiles, out, st);
        case MR_F16:
            return cone ? mr::launch_bp<MR_CONE, __half>(ring, views, grids, tiles, n_tiles, out, st)
                        : mr::launch_bp<MR_PARALLEL, __half>(ring, views, grids, tiles, n_tiles, out, st);
        default:
            return MR_ERR_INVALID;
    }
}
