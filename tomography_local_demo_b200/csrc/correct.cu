// Raw detector counts -> line integrals, without the filter: the correction of the scan
// loaders (minirecast flexray.py:111-116 + 174-184, hdf5.py:24-31 + 73-78) for callers that
// want the corrected projection stack itself, with the loaders' detector crop.
//
// One thread per output pixel, consecutive threads along detector columns (coalesced
// stores; each thread reads its bin x bin block of raw counts). HBM-bound.
#include "mr_common.cuh"

namespace mr {

constexpr int CORR_TX = 128;

template <int MODE>
__global__ void __launch_bounds__(CORR_TX)
correct_u16_kernel(const uint16_t* __restrict__ raw, long long s_view, long long s_row, int bin, int flip,
                   int rows_full, int row0, int col0, int rows, int cols, const float* __restrict__ dark,
                   const float* __restrict__ scale, long long s_frame, float* __restrict__ out, long long so_row,
                   long long so_view) {
    const int c = blockIdx.x * CORR_TX + threadIdx.x;
    const int r = blockIdx.y;
    const int v = blockIdx.z;
    if (c >= cols) return;
    const int y = r + row0;                                 // row of the full binned frame
    const int ys = flip ? rows_full - 1 - y : y;            // the same row in raw orientation
    const int x = c + col0;
    const uint16_t* p = raw + (long long)v * s_view + (long long)ys * bin * s_row + (long long)x * bin;
    float b;
    if (bin == 1) {
        b = (float)p[0];
    } else {
        unsigned int sum = 0;                               // <= 16 * 16 * 65535 < 2^24: exact
        for (int i = 0; i < bin; ++i)
            for (int j = 0; j < bin; ++j) sum += p[(long long)i * s_row + j];
        if (MODE == MR_CORRECT_FLEXRAY)
            b = __fdiv_rn((float)sum, (float)(bin * bin));            // float32 mean
        else
            b = __double2float_rn(__ddiv_rn((double)sum, (double)(bin * bin)));   // float64 mean -> f32
    }
    const long long f = (long long)y * s_frame + x;
    const float d = __fsub_rn(b, dark[f]);
    float t = MODE == MR_CORRECT_FLEXRAY ? __fmul_rn(d, scale[f]) : __fdiv_rn(d, scale[f]);
    t = fmaxf(t, 1e-3f);
    out[(long long)r * so_row + (long long)v * so_view + c] = -logf(t);
}

}  // namespace mr

extern "C" int mr_correct_u16(const uint16_t* raw, int64_t s_view, int64_t s_row, int32_t k, int32_t bin,
                              int32_t flip_rows, int32_t rows_full, int32_t row0, int32_t col0, int32_t rows,
                              int32_t cols, const float* dark, const float* scale, int64_t s_frame, int32_t mode,
                              float* out, int64_t so_row, int64_t so_view, void* stream) {
    if (!raw || !dark || !scale || !out) return MR_ERR_INVALID;
    if (k < 0 || rows < 0 || cols < 0 || bin < 1 || bin > 16 || rows_full < 1) return MR_ERR_INVALID;
    if (mode != MR_CORRECT_FLEXRAY && mode != MR_CORRECT_HDF5) return MR_ERR_INVALID;
    if (row0 < 0 || col0 < 0 || row0 + rows > rows_full || col0 + cols > s_frame) return MR_ERR_INVALID;
    if (s_row < (int64_t)(col0 + cols) * bin || s_view < (int64_t)rows_full * bin * s_row) return MR_ERR_INVALID;
    if (k > 65535 || rows > 65535) return MR_ERR_INVALID;
    if (k == 0 || rows == 0 || cols == 0) return MR_OK;
    const dim3 grid((unsigned)((cols + mr::CORR_TX - 1) / mr::CORR_TX), (unsigned)rows, (unsigned)k);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (mode == MR_CORRECT_FLEXRAY)
        mr::correct_u16_kernel<MR_CORRECT_FLEXRAY><<<grid, mr::CORR_TX, 0, st>>>(
            raw, (long long)s_view, (long long)s_row, bin, flip_rows, rows_full, row0, col0, rows, cols, dark, scale,
            (long long)s_frame, out, (long long)so_row, (long long)so_view);
    else
        mr::correct_u16_kernel<MR_CORRECT_HDF5><<<grid, mr::CORR_TX, 0, st>>>(
            raw, (long long)s_view, (long long)s_row, bin, flip_rows, rows_full, row0, col0, rows, cols, dark, scale,
            (long long)s_frame, out, (long long)so_row, (long long)so_view);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
