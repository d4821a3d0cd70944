// Derivatives of the back-projection f = B(q; shift, tilt) for the differentiable
// back-projector (no counterpart in minirecast; the forward operator is recon.py:156-219).
//
//   mr_project_adjoint : grad_q = B^T g - the matched forward projector: every sample's
//                        upstream gradient g[p] is scattered to the same four bilinear taps,
//                        with the same weights, that the forward kernel gathers from (the
//                        exact transpose, taps outside the detector dropped as in forward).
//   mr_backproject_matched : the forward B q with exactly the coordinate arithmetic of
//                        the two kernels below (its transpose is mr_project_adjoint to
//                        the last rounding of the sums);
//   mr_bp_grad_geom    : d<g, f>/d shift and d<g, f>/d tilt per grid, from the analytic
//                        derivative of the bilinear interpolant:
//                          dv/dcol = (1-fr)(q01-q00) + fr (q11-q10)
//                          dv/drow = (1-fc)(q10-q00) + fc (q11-q01)
//                        with dcol/dshift = 1, drow/dshift = uv, dcol/dtilt = row - shift uv - cr,
//                        drow/dtilt = -(col - shift - cc); the distance weight depends on neither.
// Geometry is recomputed from the per-view maps (nothing from the forward pass is stored).
//
// A tile's views may be split over a thread-block cluster of up to 8 CTAs (few tiles: the
// calibration's slices are a few dozen tiles): each CTA takes a contiguous share of the
// views; forward partial sums are reduced through distributed shared memory in rank order
// (deterministic, no scratch), geometry partials go through the FP64 atomics that already
// combine the tiles, and adjoint taps are scattered atomically either way.
#include <cooperative_groups.h>

#include "mr_common.cuh"

namespace cg = cooperative_groups;

namespace mr {

constexpr int GR_THREADS = 256;
constexpr int GR_PPT = 4;
constexpr int GR_VCH = 128;

enum : int { GRAD_ADJOINT = 0, GRAD_GEOM = 1, GRAD_FORWARD = 2 };

template <int KIND, int MODE, typename T>
__global__ void __launch_bounds__(GR_THREADS)
bp_grad_kernel(const T* __restrict__ ring, float* __restrict__ gring, int R, int C, int pitch,
               long long slot_stride, int n_slots, const mr_view* __restrict__ views,
               const mr_grid* __restrict__ grids,
               const mr_tile* __restrict__ tiles, const float* __restrict__ gout, double* __restrict__ dgeom) {
    __shared__ float4 s_u[GR_VCH], s_v[GR_VCH], s_w[GR_VCH];
    __shared__ float s_q[GR_VCH], s_uv[GR_VCH];
    __shared__ mr_grid s_g;
    __shared__ double s_red[2][GR_THREADS / 32];
    __shared__ float4 s_part[GR_THREADS];
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    const mr_tile t = tiles[blockIdx.x / csize];
    const int tid = threadIdx.x;
    if (tid < (int)(sizeof(mr_grid) / 4))
        reinterpret_cast<int*>(&s_g)[tid] = reinterpret_cast<const int*>(grids + t.grid)[tid];
    __syncthreads();
    const mr_grid& g = s_g;
    const bool pts = (g.flags & MR_GRID_POINTS) != 0;
    const int warp = tid >> 5, lane = tid & 31;
    const int tx = ((warp & 3) << 3) | (lane & 7);
    const int ty = ((warp >> 2) << 4) | (lane >> 3);

    float px[GR_PPT], py[GR_PPT], pz[GR_PPT], gp[GR_PPT], acc[GR_PPT];
    long long oidx[GR_PPT];
    bool live[GR_PPT];
#pragma unroll
    for (int p = 0; p < GR_PPT; ++p) {
        int i, j;
        long long o;
        bool ok;
        if (pts) {
            i = 0;
            j = t.j0 + tid + GR_THREADS * p;
            ok = j < g.n_j;
            o = g.out_offset + (long long)j * g.out_stride_j;
        } else {
            i = t.i0 + ty + 4 * p;
            j = t.j0 + tx;
            ok = i < g.n_i && j < g.n_j;
            o = g.out_offset + (long long)i * g.out_stride_i + (long long)j * g.out_stride_j +
                (long long)t.k * g.out_stride_k;
        }
        bool inside = ok;
        if (ok && !pts && (g.flags & MR_GRID_MASK_BOX)) {
            const double aj = __dmul_rn((double)j - g.mask_half, g.mask_delta);
            const double ai = __dmul_rn((double)i - g.mask_half, g.mask_delta);
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const double q = __dadd_rn(__dadd_rn(g.mask_c[e], __dmul_rn(aj, g.mask_ej[e])),
                                           __dmul_rn(ai, g.mask_ei[e]));
                inside = inside && (fabs(q) <= g.box[e]);
            }
        }
        live[p] = inside;
        oidx[p] = o;
        acc[p] = 0.f;
        gp[p] = (MODE != GRAD_FORWARD && inside) ? gout[o] * g.scale : 0.f;
        if (pts) {
            const int jj = ok ? j : 0;
            px[p] = g.points[3 * jj];
            py[p] = g.points[3 * jj + 1];
            pz[p] = g.points[3 * jj + 2];
        } else {
            px[p] = g.origin[0] + i * g.step_i[0] + j * g.step_j[0] + t.k * g.step_k[0];
            py[p] = g.origin[1] + i * g.step_i[1] + j * g.step_j[1] + t.k * g.step_k[1];
            pz[p] = g.origin[2] + i * g.step_i[2] + j * g.step_j[2] + t.k * g.step_k[2];
        }
    }
    const float shift = g.cor_shift;
    const float cc = 0.5f * (float)(C - 1), cr = 0.5f * (float)(R - 1);
    float ds = 0.f, dt = 0.f;
    int first, nv;                      // slots [first, first + nv)
    grid_view_range(g.view_begin, g.n_views, n_slots, &first, &nv);
    {                                   // this CTA's share of them
        const int b = first + (int)(((long long)nv * crank) / csize);
        const int e = first + (int)(((long long)nv * (crank + 1)) / csize);
        first = b;
        nv = e - b;
    }
    for (int v0 = 0; v0 < nv; v0 += GR_VCH) {
        const int nch = min(GR_VCH, nv - v0);
        __syncthreads();
        if (tid < nch) {
            const mr_view V = views[first + v0 + tid];
            float pu[4], pv[4];
            view_map(V, g, R, C, pu, pv);
            s_u[tid] = make_float4(pu[0], pu[1], pu[2], pu[3]);
            s_v[tid] = make_float4(pv[0], pv[1], pv[2], pv[3]);
            s_w[tid] = make_float4(V.pw[0], V.pw[1], V.pw[2], V.pw[3]);
            s_q[tid] = V.qscale;
            s_uv[tid] = V.uv;
        }
        __syncthreads();
        for (int vv = 0; vv < nch; ++vv) {
            const float4 cu = s_u[vv], cv = s_v[vv], cw = s_w[vv];
            const float qs = s_q[vv], uv = s_uv[vv];
            const long long slot = (long long)(first + v0 + vv) * slot_stride;
#pragma unroll
            for (int p = 0; p < GR_PPT; ++p) {
                if (MODE == GRAD_FORWARD ? !live[p] : gp[p] == 0.f) continue;
                float col = fmaf(cu.x, px[p], fmaf(cu.y, py[p], fmaf(cu.z, pz[p], cu.w)));
                float row = fmaf(cv.x, px[p], fmaf(cv.y, py[p], fmaf(cv.z, pz[p], cv.w)));
                float w = qs;
                if (KIND == MR_CONE) {
                    const float r = rcp_approx(fmaf(cw.x, px[p], fmaf(cw.y, py[p], fmaf(cw.z, pz[p], cw.w))));
                    col *= r;
                    row *= r;
                    w *= r * r;
                }
                const float rowc = fminf(fmaxf(row, -2.f), (float)R + 1.f);
                const float colc = fminf(fmaxf(col, -2.f), (float)C + 1.f);
                const float r0f = floorf(rowc), c0f = floorf(colc);
                const float fr = rowc - r0f, fc = colc - c0f;
                const int r0 = (int)r0f, c0 = (int)c0f;
                const bool ri0 = (unsigned)r0 < (unsigned)R, ri1 = (unsigned)(r0 + 1) < (unsigned)R;
                const bool ci0 = (unsigned)c0 < (unsigned)C, ci1 = (unsigned)(c0 + 1) < (unsigned)C;
                const long long base = slot + (long long)r0 * pitch + c0;
                if (MODE == GRAD_FORWARD) {
                    const float q00 = (ri0 && ci0) ? ld_elem(ring + base) : 0.f;
                    const float q01 = (ri0 && ci1) ? ld_elem(ring + base + 1) : 0.f;
                    const float q10 = (ri1 && ci0) ? ld_elem(ring + base + pitch) : 0.f;
                    const float q11 = (ri1 && ci1) ? ld_elem(ring + base + pitch + 1) : 0.f;
                    const float a = fmaf(fc, q01 - q00, q00);
                    const float b = fmaf(fc, q11 - q10, q10);
                    acc[p] = fmaf(w, fmaf(fr, b - a, a), acc[p]);
                } else if (MODE == GRAD_ADJOINT) {
                    const float a = w * gp[p];
                    if (ri0 && ci0) atomicAdd(gring + base, a * (1.f - fr) * (1.f - fc));
                    if (ri0 && ci1) atomicAdd(gring + base + 1, a * (1.f - fr) * fc);
                    if (ri1 && ci0) atomicAdd(gring + base + pitch, a * fr * (1.f - fc));
                    if (ri1 && ci1) atomicAdd(gring + base + pitch + 1, a * fr * fc);
                } else {
                    const float q00 = (ri0 && ci0) ? ld_elem(ring + base) : 0.f;
                    const float q01 = (ri0 && ci1) ? ld_elem(ring + base + 1) : 0.f;
                    const float q10 = (ri1 && ci0) ? ld_elem(ring + base + pitch) : 0.f;
                    const float q11 = (ri1 && ci1) ? ld_elem(ring + base + pitch + 1) : 0.f;
                    // the clamped coordinate has zero slope outside [-2, C+1] x [-2, R+1]
                    const bool live_c = col == colc, live_r = row == rowc;
                    const float dcol = live_c ? fmaf(fr, q11 - q10, (1.f - fr) * (q01 - q00)) : 0.f;
                    const float drow = live_r ? fmaf(fc, q11 - q01, (1.f - fc) * (q10 - q00)) : 0.f;
                    const float a = w * gp[p];
                    ds = fmaf(a, fmaf(drow, uv, dcol), ds);
                    dt = fmaf(a, dcol * (row - shift * uv - cr) - drow * (col - shift - cc), dt);
                }
            }
        }
    }
    if (MODE == GRAD_FORWARD && csize > 1) {
        s_part[tid] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        cluster.sync();
        if (crank == 0) {
            for (int r = 1; r < csize; ++r) {
                const float4 o = cluster.map_shared_rank(s_part, r)[tid];
                acc[0] += o.x; acc[1] += o.y; acc[2] += o.z; acc[3] += o.w;
            }
        }
    }
    if (MODE == GRAD_FORWARD && crank == 0) {
#pragma unroll
        for (int p = 0; p < GR_PPT; ++p) {
            const bool ok = pts ? (t.j0 + tid + GR_THREADS * p < g.n_j)
                                : (t.i0 + ty + 4 * p < g.n_i && t.j0 + tx < g.n_j);
            if (ok) {
                const float val = live[p] ? acc[p] * g.scale : 0.f;
                gring[oidx[p]] = g.accumulate ? gring[oidx[p]] + val : val;
            }
        }
    }
    if (MODE == GRAD_GEOM) {
        double a = ds, b = dt;
        for (int o = 16; o; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) { s_red[0][warp] = a; s_red[1][warp] = b; }
        __syncthreads();
        if (tid == 0) {
            double sa = 0.0, sb = 0.0;
            for (int w = 0; w < GR_THREADS / 32; ++w) { sa += s_red[0][w]; sb += s_red[1][w]; }
            atomicAdd(dgeom + 2 * t.grid, sa);
            atomicAdd(dgeom + 2 * t.grid + 1, sb);
        }
    }
    if (MODE == GRAD_FORWARD && csize > 1) cluster.sync();   // partials stay alive until read
}

template <int KIND, int MODE, typename T>
static int launch_grad(const mr_ring* ring, float* gring, const mr_view* views, const mr_grid* grids,
                       const mr_tile* tiles, int64_t n_tiles, const float* gout, double* dgeom, cudaStream_t st) {
    // CTAs per tile: enough for about four waves of CTAs on the GPU, at most 8 (portable cluster)
    int dev = 0, sms = 148;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int cl = 1;
    while (cl < 8 && n_tiles * cl < 4LL * sms) cl *= 2;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(GR_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int64_t max_chunk = 2147483647LL / cl;
    for (int64_t t0 = 0; t0 < n_tiles; t0 += max_chunk) {
        const int64_t n = (n_tiles - t0) < max_chunk ? (n_tiles - t0) : max_chunk;
        cfg.gridDim = dim3((unsigned)(n * cl));
        MR_CUDA_TRY(cudaLaunchKernelEx(&cfg, bp_grad_kernel<KIND, MODE, T>, static_cast<const T*>(ring->data), gring,
                                       ring->rows, ring->cols, ring->col_pitch, (long long)ring->slot_stride,
                                       (int)ring->n_slots, views, grids, tiles + t0, gout, dgeom));
    }
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

static int check_ring(const mr_ring* ring) {
    if (!ring || !ring->data) return MR_ERR_INVALID;
    if (ring->rows <= 0 || ring->cols <= 0 || ring->col_pitch < ring->cols) return MR_ERR_INVALID;
    if (ring->slot_stride < (int64_t)ring->rows * ring->col_pitch) return MR_ERR_INVALID;
    if (ring->kind != MR_CONE && ring->kind != MR_PARALLEL) return MR_ERR_INVALID;
    return MR_OK;
}

}  // namespace mr

extern "C" int mr_project_adjoint(const mr_ring* grad_ring, const mr_view* views, const mr_grid* grids,
                                  const mr_tile* tiles, int64_t n_tiles, const float* grad_out, void* stream) {
    int rc = mr::check_ring(grad_ring);
    if (rc != MR_OK) return rc;
    if (grad_ring->dtype != MR_F32 || !views || !grids || !grad_out || n_tiles < 0) return MR_ERR_INVALID;
    if (n_tiles > 0 && !tiles) return MR_ERR_INVALID;
    if (n_tiles == 0) return MR_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* g = static_cast<float*>(grad_ring->data);
    return grad_ring->kind == MR_CONE
               ? mr::launch_grad<MR_CONE, mr::GRAD_ADJOINT, float>(grad_ring, g, views, grids, tiles, n_tiles,
                                                                  grad_out, nullptr, st)
               : mr::launch_grad<MR_PARALLEL, mr::GRAD_ADJOINT, float>(grad_ring, g, views, grids, tiles,
                                                                      n_tiles, grad_out, nullptr, st);
}

extern "C" int mr_backproject_matched(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                                      const mr_tile* tiles, int64_t n_tiles, float* out, void* stream) {
    int rc = mr::check_ring(ring);
    if (rc != MR_OK) return rc;
    if (!views || !grids || !out || n_tiles < 0 || (n_tiles > 0 && !tiles)) return MR_ERR_INVALID;
    if (n_tiles == 0) return MR_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool cone = ring->kind == MR_CONE;
    switch (ring->dtype) {
        case MR_F32:
            return cone ? mr::launch_grad<MR_CONE, mr::GRAD_FORWARD, float>(ring, out, views, grids, tiles, n_tiles,
                                                                           nullptr, nullptr, st)
                        : mr::launch_grad<MR_PARALLEL, mr::GRAD_FORWARD, float>(ring, out, views, grids, tiles,
                                                                               n_tiles, nullptr, nullptr, st);
        case MR_BF16:
            return cone ? mr::launch_grad<MR_CONE, mr::GRAD_FORWARD, __nv_bfloat16>(ring, out, views, grids, tiles,
                                                                                   n_tiles, nullptr, nullptr, st)
                        : mr::launch_grad<MR_PARALLEL, mr::GRAD_FORWARD, __nv_bfloat16>(ring, out, views, grids,
                                                                                       tiles, n_tiles, nullptr,
                                                                                       nullptr, st);
        case MR_F16:
            return cone ? mr::launch_grad<MR_CONE, mr::GRAD_FORWARD, __half>(ring, out, views, grids, tiles, n_tiles,
                                                                            nullptr, nullptr, st)
                        : mr::launch_grad<MR_PARALLEL, mr::GRAD_FORWARD, __half>(ring, out, views, grids, tiles,
                                                                                n_tiles, nullptr, nullptr, st);
        default:
            return MR_ERR_INVALID;
    }
}

extern "C" int mr_bp_grad_geom(const mr_ring* ring, const mr_view* views, const mr_grid* grids,
                               const mr_tile* tiles, int64_t n_tiles, const float* grad_out,
                               double* dgeom, void* stream) {
    int rc = mr::check_ring(ring);
    if (rc != MR_OK) return rc;
    if (!views || !grids || !grad_out || !dgeom || n_tiles < 0) return MR_ERR_INVALID;
    if (n_tiles > 0 && !tiles) return MR_ERR_INVALID;
    if (n_tiles == 0) return MR_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool cone = ring->kind == MR_CONE;
    switch (ring->dtype) {
        case MR_F32:
            return cone ? mr::launch_grad<MR_CONE, mr::GRAD_GEOM, float>(ring, nullptr, views, grids, tiles,
                                                                        n_tiles, grad_out, dgeom, st)
                        : mr::launch_grad<MR_PARALLEL, mr::GRAD_GEOM, float>(ring, nullptr, views, grids, tiles,
                                                                            n_tiles, grad_out, dgeom, st);
        case MR_BF16:
            return cone ? mr::launch_grad<MR_CONE, mr::GRAD_GEOM, __nv_bfloat16>(ring, nullptr, views, grids,
                                                                                tiles, n_tiles, grad_out, dgeom, st)
                        : mr::launch_grad<MR_PARALLEL, mr::GRAD_GEOM, __nv_bfloat16>(ring, nullptr, views, grids,
                                                                                    tiles, n_tiles, grad_out, dgeom,
                                                                                    st);
        case MR_F16:
            return cone ? mr::launch_grad<MR_CONE, mr::GRAD_GEOM, __half>(ring, nullptr, views, grids, tiles,
                                                                         n_tiles, grad_out, dgeom, st)
                        : mr::launch_grad<MR_PARALLEL, mr::GRAD_GEOM, __half>(ring, nullptr, views, grids, tiles,
                                                                             n_tiles, grad_out, dgeom, st);
        default:
            return MR_ERR_INVALID;
    }
}
