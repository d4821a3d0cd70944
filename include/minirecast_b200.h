/*
 * minirecast_b200.h - C ABI of the B200 (sm_100a) filter / back-projection library.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t passed as
 * `void*` (NULL = legacy default stream), allocates no device memory, and returns an
 * int status (MR_OK = 0, negative on error). Work is enqueued on the given stream;
 * errors found on the host (bad sizes, bad enums) are returned before anything is
 * launched. The functions keep no state between calls except immutable tables.
 *
 * Conventions (the same as minirecast, the reference):
 *   - projections are ASTRA-style; the filtered store ("ring") is [slot][row][col]
 *     with a row pitch of `col_pitch` elements, slots in arrival order;
 *   - detector centre at ((R-1)/2, (C-1)/2); bilinear taps outside [0,R)x[0,C) are 0;
 *   - a cone view's sample position p projects to
 *         col = (pu . [p,1]) / den,  row = (pv . [p,1]) / den,  den = pw . [p,1]
 *     with den = L / SOD, and its FDK distance weight is 1/den^2 = (SOD/L)^2;
 *     a parallel view has pw = (0,0,0,1) and weight 1.
 */
#ifndef MINIRECAST_B200_H
#define MINIRECAST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MR_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------- */
#define MR_OK                0
#define MR_ERR_INVALID      -1   /* bad argument, found on the host before any launch */
#define MR_ERR_CUDA         -2   /* a CUDA runtime call or launch failed */
#define MR_ERR_UNSUPPORTED  -3   /* valid but not built (e.g. FFT length out of range) */
#define MR_ERR_TIMEOUT      -4   /* a bounded device-side wait gave up */
#define MR_ERR_SCRATCH_LIMIT -5  /* the request needs more than the library's fixed device
                                    scratch (mr_backproject_persistent_noalloc) */
#define MR_ERR_CAPTURE      -6   /* the first call of mr_backproject_persistent_noalloc on a
                                    device came while its stream was being captured */

/* ---- element types ------------------------------------------------------------- */
#define MR_F32   0
#define MR_BF16  1
#define MR_F16   2
#define MR_U16   3

/* ---- beam geometry kinds ------------------------------------------------------- */
#define MR_PARALLEL 0
#define MR_CONE     1

/* Device-resident filtered-projection store. Host struct, passed by pointer. */
typedef struct mr_ring {
    void*    data;          /* device pointer to slot 0, row 0, col 0 */
    int32_t  dtype;         /* MR_F32 / MR_BF16 / MR_F16 */
    int32_t  kind;          /* MR_PARALLEL / MR_CONE */
    int32_t  rows;          /* R */
    int32_t  cols;          /* C (columns >= C inside the pitch are never read) */
    int32_t  col_pitch;     /* elements per stored row, >= C, multiple of 8 */
    int32_t  n_slots;       /* capacity in views */
    int64_t  slot_stride;   /* elements per slot, >= rows * col_pitch */
} mr_ring;

/* One stored view: FP32 projective map built on the host in FP64. 64 bytes. */
typedef struct mr_view {
    float pu[4];            /* col * den = pu . (x, y, z, 1) */
    float pv[4];            /* row * den = pv . (x, y, z, 1) */
    float pw[4];            /* den = pw . (x, y, z, 1) */
    float uv;               /* row shift per column of COR shift: (u . v) / |v|^2 */
    float qscale;           /* stored value * qscale = filtered value (1 for FP32/BF16) */
    float pad[2];
} mr_view;

/* Sample grid of one reconstruction request. 256 bytes.
 *   p(i,j,k) = origin + i*step_i + j*step_j + k*step_k   (mm, FP32)
 *   out[out_offset + i*out_stride_i + j*out_stride_j + k*out_stride_k]
 *       (+)= scale * sum_{view_begin <= v < view_begin + n_views} w_v(p) * bilinear(ring[v], row_v(p), col_v(p))
 * With MR_GRID_MASK_BOX a sample is written as 0 unless the FP64 point
 *   c + a_j*e_j + a_i*e_i,  a_x = (x - mask_half) * mask_delta
 * lies in the box (|p_x| <= box_x for every axis), evaluated in the rounding order
 * of minirecast slice_points (recon.py:238-265), so the mask matches it bit for bit.
 * With MR_GRID_POINTS the positions are points[j*3 + 0..2] (n_i = n_k = 1).
 * cor_shift and the tilt act on every view's projective map (see tilt_cos below). */
#define MR_GRID_MASK_BOX 1
#define MR_GRID_POINTS   2
typedef struct mr_grid {
    float   origin[3];
    float   step_i[3];
    float   step_j[3];
    float   step_k[3];
    float   cor_shift;      /* rotation-centre shift, detector columns */
    float   scale;          /* pi / n_views for FBP/FDK */
    int32_t n_i, n_j, n_k;
    int32_t n_views;        /* use slots [0, n_views) - the snapshot at admission */
    int32_t flags;
    float   tilt;           /* detector in-plane rotation (rad), informational */
    int64_t out_offset;
    int64_t out_stride_i, out_stride_j, out_stride_k;
    const float* points;    /* device, MR_GRID_POINTS only */
    float   tilt_cos, tilt_sin;   /* (0, 0) = no tilt. Detector coordinates are rotated
                                     about the detector centre (cc, cr) = ((C-1)/2, (R-1)/2):
                                     col' = cc + c (col-cc) + s (row-cr) + shift,
                                     row' = cr - s (col-cc) + c (row-cr) + shift * uv */
    double  mask_c[3];      /* plane centre */
    double  mask_ej[3];     /* unit vector along j (columns) */
    double  mask_ei[3];     /* unit vector along i (rows) */
    double  mask_half;      /* (n - 1) / 2 */
    double  mask_delta;     /* pixel size */
    double  box[3];         /* half sizes of the volume box */
    int32_t view_begin;     /* first slot summed: slots [view_begin, view_begin + n_views) */
    int32_t accumulate;     /* 0: out = result (0 outside the box); 1: out += result (a
                               partial sum over a range of views, same scale) */
    int64_t pad2;
} mr_grid;

/* One work item of a back-projection launch: a tile of one grid. 16 bytes. */
typedef struct mr_tile {
    int32_t grid;           /* index into the grid array */
    int32_t i0, j0, k;      /* first sample of the tile */
} mr_tile;

/* Per-view parameters of the ingest / filter kernels, built on the host in FP64. 32 bytes.
 * FDK cosine weight w(r,c) = sdd / sqrt(sdd^2 + a^2 + b^2), a = a0 + c*da, b = b0 + r*db;
 * sdd == 0 means no weight (parallel beam). The filter output is
 *   ring[slot][r][c] = out_scale * gain * (g * (x w))[r][c]
 * where g is the ramp kernel whose spectrum is the table H (built for tau = 1) and
 * gain = 1 / (tau * N), N the FFT length. */
typedef struct mr_filter_view {
    float   a0, da, b0, db;
    float   sdd;
    float   gain;
    float   out_scale;
    int32_t slot;
} mr_filter_view;

/* ---- library information ------------------------------------------------------- */
int         mr_abi_version(void);
const char* mr_status_string(int status);
/* Text of the CUDA error behind the last MR_ERR_CUDA returned on the calling host
 * thread ("" if none). */
const char* mr_last_cuda_error(void);
/* sizeof() of the ABI structs, for layout checks by bindings:
 * which = 0 mr_ring, 1 mr_view, 2 mr_grid, 3 mr_tile, 4 mr_filter_view; -1 otherwise. */
int         mr_struct_size(int which);
/* Samples per back-projection tile along i and j (host-side planning). */
void        mr_bp_tile_shape(int32_t* tile_i, int32_t* tile_j);

/* Host-only: split `n_grids` grids (host memory) into tiles (host memory).
 * Writes at most `capacity` tiles and returns the number needed in *n_tiles. */
int mr_plan_tiles(const mr_grid* grids_host, int32_t n_grids,
                  mr_tile* tiles_host, int64_t capacity, int64_t* n_tiles);

/* ---- back-projection ------------------------------------------------------------
 * Replaces minirecast recon.py:193-219 (bp_cone_numba, with _bil_nb 156-173) and
 * recon.py:175-191 (bp_parallel_numba) as called by reconstruct_points
 * recon.py:405-424 / reconstruct_plane 426-440 / reconstruct_volume 442-470.
 * Many grids (requests) of any size, zoom and orientation go in one launch; every
 * sample accumulates in FP32 registers over slots [0, n_views) of its grid. */
int mr_backproject(const mr_ring* ring, const mr_view* views_dev,
                   const mr_grid* grids_dev, const mr_tile* tiles_dev, int64_t n_tiles,
                   float* out_dev, void* stream);

/* Same contract as mr_backproject for regular grids (not MR_GRID_POINTS), with the
 * detector footprint of every (tile, view) staged into shared memory by the TMA unit
 * (cp.async.bulk.tensor, zero fill outside the detector) and predicate-free software
 * bilinear. The ring needs 16-byte aligned data, rows and slots. `status_dev` (may be
 * NULL) receives MR_ERR_TIMEOUT if a bounded wait on a stage ever gave up. */
int mr_backproject_staged(const mr_ring* ring, const mr_view* views_dev,
                          const mr_grid* grids_dev, const mr_tile* tiles_dev, int64_t n_tiles,
                          float* out_dev, int32_t* status_dev, void* stream);

/* Persistent form of mr_backproject_staged for serving: a fixed grid of CTA clusters
 * (as many as fit on the GPU at once, at most max_tiles) pulls tile indices from a work
 * counter until it reaches min(*n_tiles_dev, max_tiles) (device int64; max_tiles <= 2^31),
 * so the launch shape
 * does not depend on the batch and the call can be captured in a CUDA graph once and
 * replayed with new grid/tile contents. counter_dev: caller-provided 4-byte device
 * scratch (4-byte aligned), zeroed on `stream` by this call; calls that share a counter
 * must be ordered on one stream. */
int mr_backproject_persistent(const mr_ring* ring, const mr_view* views_dev,
                              const mr_grid* grids_dev, const mr_tile* tiles_dev,
                              const int64_t* n_tiles_dev, int64_t max_tiles,
                              uint32_t* counter_dev, float* out_dev, int32_t* status_dev,
                              void* stream);

/* No counterpart in the reference (minirecast runs on the CPU and never allocates device
 * memory). The same back-projection as mr_backproject_persistent, for callers that cannot
 * call cudaMalloc: a host whose device memory is handed out by another component (an
 * acquisition or frame-grabber SDK, an application-wide memory pool) and that therefore
 * owns no device buffer of its own to use as the work counter, or code on a live
 * acquisition path where an allocation could synchronise the device and stall the scan.
 * The work counter lives in the library's own device scratch: a 256-byte static array
 * (MR_NOALLOC_SCRATCH_BYTES) that every GPU which loads the library holds until the
 * process exits. Nothing is allocated by this call; the caller still passes every input
 * and output. The counter is zeroed on `stream` by each call.
 *   - The device that owns `stream` must be the current device.
 *   - The first call on a device looks up the array's device address (and may load the
 *     library's device code); make that first call before any stream capture. A first
 *     call on a stream that is being captured returns MR_ERR_CAPTURE and launches nothing.
 *   - The address is kept for the life of the process. After cudaDeviceReset (or a
 *     reset of the primary context by the host application) the array may move: do not
 *     call this entry point again in that process.
 *   - Every call on a device shares the one counter: calls that overlap on the GPU race
 *     and give wrong results. Order them on one stream (or wait between them).
 *   - max_tiles above MR_NOALLOC_MAX_TILES (the range one 32-bit counter can hand out)
 *     returns MR_ERR_SCRATCH_LIMIT before anything is launched. */
#define MR_NOALLOC_SCRATCH_BYTES 256
#define MR_NOALLOC_MAX_TILES (((int64_t)1) << 31)
int mr_backproject_persistent_noalloc(const mr_ring* ring, const mr_view* views_dev,
                                      const mr_grid* grids_dev, const mr_tile* tiles_dev,
                                      const int64_t* n_tiles_dev, int64_t max_tiles,
                                      float* out_dev, int32_t* status_dev, void* stream);

/* ---- derivatives of the back-projection (no counterpart in minirecast: the reference
 * back-projector is not differentiable; the forward operator is recon.py:156-219) ----
 * Matched forward projector, the exact transpose of mr_backproject: grad_ring (F32, the
 * ring layout, zeroed by the caller) += B^T grad_out, where grad_out has the layout of
 * the forward output. Samples masked out of the box carry no gradient. */
int mr_project_adjoint(const mr_ring* grad_ring, const mr_view* views_dev,
                       const mr_grid* grids_dev, const mr_tile* tiles_dev, int64_t n_tiles,
                       const float* grad_out_dev, void* stream);

/* The forward operator of the differentiable path: the same result as mr_backproject,
 * computed with the coordinate arithmetic of mr_project_adjoint / mr_bp_grad_geom, so
 * that the adjoint is its transpose to the rounding of the sums. */
int mr_backproject_matched(const mr_ring* ring, const mr_view* views_dev,
                           const mr_grid* grids_dev, const mr_tile* tiles_dev, int64_t n_tiles,
                           float* out_dev, void* stream);

/* dgeom[2*g + 0] += d<grad_out, f_g>/d cor_shift, dgeom[2*g + 1] += d<...>/d tilt (per
 * radian) for every grid g, with f the forward output of mr_backproject on `ring`.
 * dgeom: device doubles, zeroed by the caller. */
int mr_bp_grad_geom(const mr_ring* ring, const mr_view* views_dev, const mr_grid* grids_dev,
                    const mr_tile* tiles_dev, int64_t n_tiles, const float* grad_out_dev,
                    double* dgeom_dev, void* stream);

/* ---- filtering ---------------------------------------------------------------------
 * Replaces recon.py:85-104 (fdk_filter_block) and recon.py:58-64 (filter_rows, via
 * ramp_response 34-55) as called from add_projections recon.py:357-362.
 * Input element (v, r, c) is block[v*s_view + r*s_row + c] (f32, device); the ASTRA
 * block [rows, k, cols] of the reference has s_view = cols, s_row = k*cols.
 * H: device, n_fft reals (full spectrum, mirrored), twiddle: device, n_fft complex
 * exp(-2 pi i m / n_fft) as interleaved float pairs. n_fft = 2^log2n >= 2*cols. */
int mr_filter_f32(const float* block, int64_t s_view, int64_t s_row,
                  int32_t k, const mr_filter_view* views_dev,
                  const float* H_dev, const float* twiddle_dev, int32_t log2n,
                  const mr_ring* ring, void* stream);

/* ---- fused raw ingest ----------------------------------------------------------
 * Replaces flexray.py:111-116 + 174-184 (bin, flipud, (P-D)*gain, clip 1e-3, -log)
 * and hdf5.py:24-31 + 73-78, fused with the filter above. Raw element (v, y, x) is
 * raw[v*s_view + y*s_row + x] (uint16, device). Output pixel (r, c) averages raw
 * rows [r'*bin, r'*bin+bin) x cols [c*bin, c*bin+bin) with r' = flip ? rows-1-r : r.
 * dark, gain: device f32 [rows][cols] in output orientation, already binned:
 *   x = -log(max((mean - dark) * gain, 1e-3)). */
int mr_ingest_u16(const uint16_t* raw, int64_t s_view, int64_t s_row,
                  int32_t bin, int32_t flip_rows,
                  const float* dark_dev, const float* gain_dev,
                  int32_t k, const mr_filter_view* views_dev,
                  const float* H_dev, const float* twiddle_dev, int32_t log2n,
                  const mr_ring* ring, void* stream);

/* ---- iso-surface of a volume (marching cubes) -------------------------------------
 * Replaces the contour step of model.py:40-69 (extract_surface: VTK flying edges, or
 * scikit-image's marching cubes). vol: device f32 [nx][ny][nz] (z fastest), the grid point
 * (i, j, k) at origin + spacing * (i, j, k); a corner is inside when its value > iso (NaN:
 * outside). Cells are the (nx-1)(ny-1)(nz-1) cubes in memory order of their lowest corner,
 * in blocks of up to 256 cells of one z row (nx, ny <= 65536). The case table is built by the library from the cube's geometry:
 * table[16*m + 0..14] = three edge numbers per triangle of pattern m (-1 after the last),
 * table[16*m + 15] = triangle count (<= 5); corners c = dx + 2 dy + 4 dz, edges 0-3 along
 * x from the corners with dx = 0, 4-7 along y, 8-11 along z; normals point from inside
 * to outside; a shared face is cut alike from both cells, so surfaces are closed. */
int64_t mr_mc_blocks(int32_t nx, int32_t ny, int32_t nz);     /* (nx-1)(ny-1)ceil((nz-1)/256) */
int mr_mc_table(int8_t* table_host);                          /* 256 x 16 bytes, host only */
/* block_counts: device int32 [mr_mc_blocks()], the triangles of each block. */
int mr_mc_count(const float* vol, int32_t nx, int32_t ny, int32_t nz, float iso,
                int32_t* block_counts_dev, void* stream);
/* block_offsets: device int64, the exclusive prefix sums of block_counts; n_tri: their
 * total (the capacity of the outputs). Per vertex v of triangle t (v = 3t + q):
 * tri_edges[v] = grid edge id 3 * ((i*ny + j)*nz + k) + axis of the edge it lies on
 * (identical for the cells sharing the edge), tri_pos[3v .. 3v+2] = its position,
 * origin + spacing * (corner + s * axis), s = (iso - v_a) / (v_b - v_a), every FP32
 * operation rounded on its own. origin: host, 3 doubles. */
int mr_mc_emit(const float* vol, int32_t nx, int32_t ny, int32_t nz, float iso,
               const double* origin, double spacing, const int64_t* block_offsets_dev,
               int64_t n_tri, int64_t* tri_edges_dev, float* tri_pos_dev, void* stream);

/* ---- raw correction alone (the scan loaders' output stack) ------------------------
 * Replaces the per-projection correction of flexray.py:111-116 + 174-184 (`corrected`,
 * mode MR_CORRECT_FLEXRAY: float32 bin mean, (mean - dark) * scale, scale = the gain
 * 1/max(F-D, 1)) and of hdf5.py:24-31 + 73-78 (mode MR_CORRECT_HDF5: float64 bin mean
 * rounded to float32, (mean - dark) / scale, scale = max(F-D, 1e-6)), then clip 1e-3 and
 * -log, with the loaders' detector crop:
 *   out[r*so_row + v*so_view + c] = -log(max(t, 1e-3)) for v < k, r < rows, c < cols,
 * t from the bin x bin mean of raw (uint16, device, view v at raw + v*s_view, row stride
 * s_row) at full binned row y = row0 + r (raw row flip ? rows_full-1-y : y, i.e. the frame
 * flipped upside down before the crop) and binned column x = col0 + c, and from
 * dark[y*s_frame + x], scale[y*s_frame + x] (device f32, the full binned frame in output
 * orientation). bin <= 16; k, rows <= 65535. */
#define MR_CORRECT_FLEXRAY 0
#define MR_CORRECT_HDF5    1
int mr_correct_u16(const uint16_t* raw, int64_t s_view, int64_t s_row, int32_t k, int32_t bin,
                   int32_t flip_rows, int32_t rows_full, int32_t row0, int32_t col0, int32_t rows,
                   int32_t cols, const float* dark_dev, const float* scale_dev, int64_t s_frame,
                   int32_t mode, float* out_dev, int64_t so_row, int64_t so_view, void* stream);

/* ---- tensor-core Toeplitz filter (the measured alternative to the FFT filter) ------
 * Same contracts as mr_filter_f32 / mr_ingest_u16 (recon.py:58-104; flexray.py:174-184 +
 * hdf5.py:73-78 for the raw correction), with the row filter computed as a GEMM on the
 * tcgen05 tensor cores: for outputs and inputs inside a row, filtering is y = T x with
 * the Toeplitz matrix T[n][j] = g[(n - j) mod n_fft], g = ifft(H) for tau = 1.
 * Operands are split into two 16-bit parts (x = x_hi + x_lo, g = g_hi + g_lo; `format`
 * MR_F16 or MR_BF16) with FP32 accumulation; the hi/lo cross terms are kept on the three
 * 64-wide block diagonals nearest the main one, where |g| is large. FP16 parts carry 22
 * bits (filtered rows within ~1e-5 of FP64), BF16 parts 16 bits (~5e-4: the ramp filter
 * cancels ~400x on smooth rows). FP16 operands are brought into range by powers of two:
 * `t_scale` (from mr_toeplitz_image) for g, `x_scale` for the inputs (the FP32 entry
 * point needs max |x| * x_scale < 2^14; the raw entry point uses 1024, since
 * |-log(max(t, 1e-3))| < 11.1).
 * Rows of at most 512 columns (MR_ERR_UNSUPPORTED beyond); col_pitch and slot_stride
 * multiples of 8 elements, 16-byte aligned ring.
 * `image_dev`: device copy of the operand built by mr_toeplitz_image (16-byte aligned).
 * `status_dev` (may be NULL) receives MR_ERR_TIMEOUT if a bounded device wait gave up. */
int64_t mr_toeplitz_image_bytes(int32_t cols);
/* Host-only: write the split Toeplitz blocks of the FP64 kernel g[0..n_fft) in `format`
 * into `image_host` (mr_toeplitz_image_bytes(cols) bytes), in the kernel's shared-memory
 * layout (SWIZZLE_128B K-major), and the power-of-two scale applied to g in *t_scale. */
int mr_toeplitz_image(const double* g, int32_t n_fft, int32_t cols, int32_t format,
                      void* image_host, float* t_scale);
int mr_filter_f32_tc(const float* block, int64_t s_view, int64_t s_row, int32_t k,
                     const mr_filter_view* views_dev, const void* image_dev, int32_t format,
                     float t_scale, float x_scale, int32_t n_fft,
                     const mr_ring* ring, int32_t* status_dev, void* stream);
int mr_ingest_u16_tc(const uint16_t* raw, int64_t s_view, int64_t s_row,
                     int32_t bin, int32_t flip_rows,
                     const float* dark_dev, const float* gain_dev,
                     int32_t k, const mr_filter_view* views_dev,
                     const void* image_dev, int32_t format, float t_scale, int32_t n_fft,
                     const mr_ring* ring, int32_t* status_dev, void* stream);

/* ---- rotation-centre search score ---------------------------------------------
 * Replaces the scoring loop of recon.py:498-519 (estimate_cor): for each of n_imgs
 * images (f32, device, image i at imgs + i*stride, n_pix pixels) the FP64 score
 * sum(p log p) of a `bins`-bin histogram of its non-zero pixels, with numpy.histogram's
 * bin assignment (range = [min, max] of the non-zero pixels, top edge inclusive).
 * scores: device, n_imgs doubles. bins <= 1024. */
int mr_slice_entropy(const float* imgs, int32_t n_imgs, int64_t stride, int32_t n_pix,
                     int32_t bins, double* scores_dev, void* stream);

/* ---- volume consumers -----------------------------------------------------------
 * The device passes of model.py:18-29 (otsu_threshold) over a reconstructed volume of
 * n f32 voxels (device, 4-byte aligned, any layout): the host computes the percentile
 * interpolation and the Otsu sums over the bins in FP64 from what these return.
 * ws: device workspace of mr_volume_workspace_bytes() bytes (8-byte aligned), shared by
 * the three calls of one threshold; calls on one workspace must not overlap. */
int64_t mr_volume_workspace_bytes(void);

/* Counts of the voxels != 0 and of the NaN voxels, and the order keys of the smallest
 * and largest non-zero, non-NaN value (key = bits | 2^31 for x >= 0, ~bits for x < 0).
 * stats_host (optional, host): {nonzero, nan, kmin | (uint64_t)kmax << 32}; when given,
 * the call waits for the stream. */
int mr_volume_stats(const float* vol, int64_t n, void* ws, uint64_t* stats_host, void* stream);

/* The values of rank ranks[j] (0-based, ascending) among the non-zero, non-NaN voxels,
 * j < n_ranks <= 4, into values_dev (device, n_ranks floats): exact order statistics
 * (a radix select over the bits in which kmin and kmax, from mr_volume_stats, differ). */
int mr_volume_select(const float* vol, int64_t n, const int64_t* ranks_host, int32_t n_ranks,
                     uint32_t kmin, uint32_t kmax, void* ws, float* values_dev, void* stream);

/* hist_dev[b] (device, bins uint64, overwritten) = the number of non-zero, non-NaN voxels
 * whose FP64 value clipped to [lo, hi] falls in bin b of numpy.histogram(..., bins,
 * range=(lo, hi)): edges_dev (device, bins + 1 doubles) = np.linspace(first, last,
 * bins + 1) with (first, last) = (lo, hi), widened by 0.5 on each side if lo == hi; a value
 * on an inner edge counts in the bin above it, the top edge in the last bin. bins <= 2048. */
int mr_volume_histogram(const float* vol, int64_t n, const double* edges_dev, int32_t bins,
                        double lo, double hi, uint64_t* hist_dev, void* stream);

/* ---- pre-processing on arrival (block layout [rows, k, cols], f32, device) ------
 * Replaces preprocess.py:31-56 (rotate_projections): every projection rotated by
 * `degrees` about the detector centre, bilinear, zero outside. in != out. */
int mr_rotate_f32(const float* in, float* out, int32_t rows, int32_t k, int32_t cols,
                  double degrees, void* stream);

/* Replaces one axis of preprocess.py:8-28 (gaussian_blur): edge padding by `pad`,
 * circular convolution over the padded length with the even kernel taps[0..n_taps-1]
 * (taps[m] = g[m] = g[-m]), crop. axis = 0 (rows) or 2 (cols). in != out. */
int mr_gaussian_axis_f32(const float* in, float* out, int32_t rows, int32_t k, int32_t cols,
                         int32_t axis, int32_t pad, const float* taps, int32_t n_taps,
                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MINIRECAST_B200_H */
