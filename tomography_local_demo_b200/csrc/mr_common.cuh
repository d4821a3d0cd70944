// Shared device helpers of the sm_100a filter / back-projection library.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "minirecast_b200.h"

namespace mr {
// The CUDA error behind the last MR_ERR_CUDA returned on this host thread.
void set_last_cuda_error(cudaError_t e);
}  // namespace mr

#define MR_CUDA_TRY(expr)                                  \
    do {                                                   \
        cudaError_t e_ = (expr);                           \
        if (e_ != cudaSuccess) {                           \
            mr::set_last_cuda_error(e_);                   \
            return MR_ERR_CUDA;                            \
        }                                                  \
    } while (0)

namespace mr {

// Stored-element loads through the read-only path, widened to FP32.
// Slots a grid sums: [first, first + count) = [view_begin, view_begin + n_views) clamped
// to the ring's n_slots, so that a descriptor running past the ring reads nothing outside it.
__device__ __forceinline__ void grid_view_range(int view_begin, int n_views, int n_slots, int* first,
                                                int* count) {
    const int b = min(max(view_begin, 0), max(n_slots, 0));
    *first = b;
    *count = max(min(n_views, n_slots - b), 0);
}

__device__ __forceinline__ float ld_elem(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ld_elem(const __nv_bfloat16* p) {
    const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
    return __uint_as_float(static_cast<unsigned>(u) << 16);
}
__device__ __forceinline__ float ld_elem(const __half* p) { return __half2float(__ldg(p)); }

// Stored-element writes from FP32 (round to nearest even).
__device__ __forceinline__ void st_elem(float* p, float v) { *p = v; }
__device__ __forceinline__ void st_elem(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void st_elem(__half* p, float v) { *p = __float2half_rn(v); }

// Fast reciprocal (PTX rcp.approx: at most 1 ulp from the correctly rounded value).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Complex arithmetic on (re, im) pairs with the packed f32x2 instructions of sm_100: each
// component is exactly the scalar operation it replaces (a - b is fma(b, -1, a), one
// rounding of the exact difference), so results are unchanged and the issue slots halve.
//   a b = (a.x b.x - a.y b.y, a.x b.y + a.y b.x) = a.x (b.x, b.y) + a.y (-b.y, b.x)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return __ffma2_rn(make_float2(a.x, a.x), b, __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x)));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

// Per-view projective map with the grid's COR shift and detector tilt applied:
//   no tilt: pu' = pu + shift pw,  pv' = pv + shift uv pw                 (recon.py:420)
//   tilt   : (col, row) rotated by the tilt about the detector centre, then shifted.
__device__ __forceinline__ void view_map(const mr_view& V, const mr_grid& g, int R, int C, float* pu,
                                         float* pv) {
    const float shift = g.cor_shift;
    if (g.tilt_cos == 0.f && g.tilt_sin == 0.f) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            pu[e] = fmaf(shift, V.pw[e], V.pu[e]);
            pv[e] = fmaf(shift * V.uv, V.pw[e], V.pv[e]);
        }
    } else {
        const float c = g.tilt_cos, s = g.tilt_sin;
        const float cc = 0.5f * (float)(C - 1), cr = 0.5f * (float)(R - 1);
        const float ku = cc * (1.f - c) - cr * s + shift;
        const float kv = cr * (1.f - c) + cc * s + shift * V.uv;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            pu[e] = fmaf(c, V.pu[e], fmaf(s, V.pv[e], ku * V.pw[e]));
            pv[e] = fmaf(-s, V.pu[e], fmaf(c, V.pv[e], kv * V.pw[e]));
        }
    }
}

}  // namespace mr
