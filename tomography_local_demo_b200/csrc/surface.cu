// Iso-surface of a reconstructed volume by marching cubes: the contour step of minirecast
// model.py:40-69 (extract_surface), which the reference hands to VTK's flying edges (or
// scikit-image). Two passes over the cells of a float32 volume [nx][ny][nz] (z fastest):
//   mr_mc_count  triangles per block of up to 256 cells of one z row (the host scans these
//                into offsets)
//   mr_mc_emit   each cell's triangles at its block's offset + its rank inside the block:
//                per vertex the grid edge it lies on (for sharing vertices between cells)
//                and its position, interpolated in FP32 along the edge
// The case table is built here from the cube's geometry (the rule is described at
// build_table) and kept in constant memory, uploaded once per device; mr_mc_table hands it
// to the host so that a binding (and the tests) can check it.
#include <cmath>
#include <mutex>

#include "mr_common.cuh"

namespace mr {

constexpr int MC_THREADS = 256;
constexpr int MC_MAX_TRI = 5;

__constant__ int8_t c_mc_tri[256][16];          // 3 edges per triangle, -1 padding; [15] = count
__constant__ int8_t c_mc_edge[12][2];           // corners of each edge (second = first + 2^axis)

// Corners c = dx + 2 dy + 4 dz; edges 0-3 along axis 0 (from the corners with dx = 0),
// 4-7 along axis 1, 8-11 along axis 2. Per inside/outside pattern (inside: value > iso),
// every cube face is walked counter-clockwise as seen from outside; each edge where the
// walk leaves the inside corners is joined to the edge where that run of inside corners
// began, and on a face whose two inside corners are diagonal (ambiguous) each inside
// corner is cut off alone. The rule depends on the face alone, so neighbouring cells cut
// a shared face alike and the surface closes. The joined segments form loops; each loop,
// reversed, is fanned into triangles whose normals point from inside to outside, from the
// first vertex whose diagonals stay off the cube faces (a diagonal on a face would touch
// the neighbouring cell's surface along it).
static void build_table(int8_t tri[256][16], int8_t edge[12][2]) {
    int ec[12][2], ne = 0;
    for (int a = 0; a < 3; ++a)
        for (int c0 = 0; c0 < 8; ++c0)
            if (!((c0 >> a) & 1)) { ec[ne][0] = c0; ec[ne][1] = c0 | (1 << a); ++ne; }
    auto edge_of = [&](int p, int q) {
        for (int e = 0; e < 12; ++e)
            if ((ec[e][0] == p && ec[e][1] == q) || (ec[e][0] == q && ec[e][1] == p)) return e;
        return -1;
    };
    int faces[6][4];
    for (int a = 0, f = 0; a < 3; ++a)
        for (int side = 0; side < 2; ++side, ++f) {
            int cs[4], n = 0;
            for (int c = 0; c < 8; ++c)
                if (((c >> a) & 1) == side) cs[n++] = c;
            double nrm[3] = {0, 0, 0}, u[3] = {0, 0, 0}, v[3];
            nrm[a] = side ? 1.0 : -1.0;
            u[(a + 1) % 3] = 1.0;
            v[0] = nrm[1] * u[2] - nrm[2] * u[1];
            v[1] = nrm[2] * u[0] - nrm[0] * u[2];
            v[2] = nrm[0] * u[1] - nrm[1] * u[0];
            double ang[4];
            for (int i = 0; i < 4; ++i) {
                double p[3] = {(double)(cs[i] & 1) - 0.5, (double)((cs[i] >> 1) & 1) - 0.5,
                               (double)((cs[i] >> 2) & 1) - 0.5};
                p[a] = 0.0;
                ang[i] = std::atan2(p[0] * v[0] + p[1] * v[1] + p[2] * v[2], p[0] * u[0] + p[1] * u[1] + p[2] * u[2]);
            }
            for (int i = 0; i < 4; ++i)                         // sort by angle
                for (int j = i + 1; j < 4; ++j)
                    if (ang[j] < ang[i]) {
                        std::swap(ang[i], ang[j]);
                        std::swap(cs[i], cs[j]);
                    }
            for (int i = 0; i < 4; ++i) faces[f][i] = cs[i];
        }
    int eface[12] = {0};                                        // faces holding each edge (bits)
    for (int e = 0; e < 12; ++e)
        for (int f = 0; f < 6; ++f) {
            int hits = 0;
            for (int i = 0; i < 4; ++i) hits += (faces[f][i] == ec[e][0]) + (faces[f][i] == ec[e][1]);
            if (hits == 2) eface[e] |= 1 << f;
        }
    for (int m = 0; m < 256; ++m) {
        int nxt[12];
        for (int e = 0; e < 12; ++e) nxt[e] = -1;
        for (int f = 0; f < 6; ++f) {
            const int* cs = faces[f];
            int in[4];
            for (int i = 0; i < 4; ++i) in[i] = (m >> cs[i]) & 1;
            const bool amb = in[0] + in[1] + in[2] + in[3] == 2 && in[0] == in[2];
            for (int i = 0; i < 4; ++i) {
                if (!(in[i] && !in[(i + 1) % 4])) continue;
                int j = i;
                if (!amb)
                    while (in[(j + 3) % 4]) j = (j + 3) % 4;
                nxt[edge_of(cs[i], cs[(i + 1) % 4])] = edge_of(cs[(j + 3) % 4], cs[j]);
            }
        }
        int out[3 * MC_MAX_TRI], nt = 0;
        bool seen[12] = {false};
        for (int e0 = 0; e0 < 12; ++e0) {
            if (nxt[e0] < 0 || seen[e0]) continue;
            int loop[12], n = 0, e = e0;
            do {
                loop[n++] = e;
                seen[e] = true;
                e = nxt[e];
            } while (e != e0);
            for (int i = 0; i < n / 2; ++i) std::swap(loop[i], loop[n - 1 - i]);
            // fan apex: the first vertex none of whose diagonals lies on a cube face
            int r = 0;
            for (; r < n; ++r) {
                bool on_face = false;
                for (int i = 2; i < n - 1; ++i)
                    if (eface[loop[r]] & eface[loop[(r + i) % n]]) on_face = true;
                if (!on_face) break;
            }
            if (r == n) r = 0;
            for (int i = 1; i + 1 < n && nt < MC_MAX_TRI; ++i) {
                out[3 * nt] = loop[r];
                out[3 * nt + 1] = loop[(r + i) % n];
                out[3 * nt + 2] = loop[(r + i + 1) % n];
                ++nt;
            }
        }
        for (int i = 0; i < 16; ++i) tri[m][i] = -1;
        for (int i = 0; i < 3 * nt; ++i) tri[m][i] = (int8_t)out[i];
        tri[m][15] = (int8_t)nt;
    }
    for (int e = 0; e < 12; ++e) {
        edge[e][0] = (int8_t)ec[e][0];
        edge[e][1] = (int8_t)ec[e][1];
    }
}

static std::once_flag g_table_once;
static int8_t g_tri[256][16], g_edge[12][2];
static std::mutex g_upload_mutex;
static bool g_uploaded[64];

static int ensure_table() {
    std::call_once(g_table_once, [] { build_table(g_tri, g_edge); });
    int dev = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return MR_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_upload_mutex);
    if (!g_uploaded[dev]) {
        MR_CUDA_TRY(cudaMemcpyToSymbol(c_mc_tri, g_tri, sizeof(g_tri)));
        MR_CUDA_TRY(cudaMemcpyToSymbol(c_mc_edge, g_edge, sizeof(g_edge)));
        g_uploaded[dev] = true;
    }
    return MR_OK;
}

struct McArgs {
    const float* vol;
    int nx, ny, nz;
    int kchunks;                                // blocks of 256 cells along z per (i, j) row
    long long cells;
    float iso;
    float ox, oy, oz, h;
};

// Cell (i, j, k) of this thread: blocks run over rows of cells along z (blockIdx.x: 256-cell
// chunk of the row, blockIdx.y: j, blockIdx.z: i), so block order is cell memory order.
// Returns the case of the cell, or -1 past the row's end.
__device__ __forceinline__ int cell_case(const McArgs& g, int& i, int& j, int& k, float val[8]) {
    i = blockIdx.z;
    j = blockIdx.y;
    k = blockIdx.x * MC_THREADS + threadIdx.x;
    if (k >= g.nz - 1) return -1;
    const float* p = g.vol + ((long long)i * g.ny + j) * g.nz + k;
    const long long sx = (long long)g.ny * g.nz, sy = g.nz;
    int m = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        val[c] = __ldg(p + (c & 1) * sx + ((c >> 1) & 1) * sy + ((c >> 2) & 1));
        m |= (val[c] > g.iso ? 1 : 0) << c;
    }
    return m;
}

__device__ __forceinline__ long long block_id(const McArgs& g) {
    return ((long long)blockIdx.z * gridDim.y + blockIdx.y) * g.kchunks + blockIdx.x;
}

__global__ void __launch_bounds__(MC_THREADS) mc_count_kernel(McArgs g, int* __restrict__ block_counts) {
    __shared__ int warp_sum[MC_THREADS / 32];
    int i, j, k;
    float val[8];
    const int m = cell_case(g, i, j, k, val);
    int cnt = m >= 0 ? c_mc_tri[m][15] : 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < MC_THREADS / 32; ++w) s += warp_sum[w];
        block_counts[block_id(g)] = s;
    }
}

__global__ void __launch_bounds__(MC_THREADS)
mc_emit_kernel(McArgs g, const long long* __restrict__ block_offsets, long long n_tri,
               long long* __restrict__ tri_edges, float* __restrict__ tri_pos) {
    __shared__ int warp_sum[MC_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int i, j, k;
    float val[8];
    const int m = cell_case(g, i, j, k, val);
    const int cnt = m >= 0 ? c_mc_tri[m][15] : 0;
    // exclusive rank of this cell's triangles inside the block
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += warp_sum[w];
    const long long first = block_offsets[block_id(g)] + before + incl - cnt;
    for (int t = 0; t < cnt; ++t) {
        const long long o = first + t;
        if (o >= n_tri) break;                          // never write past the caller's buffers
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int e = c_mc_tri[m][3 * t + q];
            const int a = c_mc_edge[e][0], b = c_mc_edge[e][1];
            const int axis = (b - a) == 1 ? 0 : ((b - a) == 2 ? 1 : 2);
            const int ia = i + (a & 1), ja = j + ((a >> 1) & 1), ka = k + ((a >> 2) & 1);
            // FP32, each operation rounded on its own: t = (iso - va) / (vb - va)
            const float s = __fdiv_rn(__fsub_rn(g.iso, val[a]), __fsub_rn(val[b], val[a]));
            float cx = (float)ia, cy = (float)ja, cz = (float)ka;
            if (axis == 0) cx = __fadd_rn(cx, s);
            else if (axis == 1) cy = __fadd_rn(cy, s);
            else cz = __fadd_rn(cz, s);
            const long long vtx = 3 * o + q;
            tri_edges[vtx] = (((long long)ia * g.ny + ja) * g.nz + ka) * 3 + axis;
            tri_pos[3 * vtx + 0] = __fadd_rn(g.ox, __fmul_rn(g.h, cx));
            tri_pos[3 * vtx + 1] = __fadd_rn(g.oy, __fmul_rn(g.h, cy));
            tri_pos[3 * vtx + 2] = __fadd_rn(g.oz, __fmul_rn(g.h, cz));
        }
    }
}

static int fill_args(McArgs& g, const float* vol, int32_t nx, int32_t ny, int32_t nz, float iso) {
    if (!vol || nx < 2 || ny < 2 || nz < 2 || !(iso == iso)) return MR_ERR_INVALID;
    if (((uintptr_t)vol & 3u)) return MR_ERR_INVALID;
    if (nx - 1 > 65535 || ny - 1 > 65535) return MR_ERR_UNSUPPORTED;     // grid y / z limits
    g.vol = vol;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.kchunks = (nz - 1 + MC_THREADS - 1) / MC_THREADS;
    g.cells = (long long)(nx - 1) * (ny - 1) * (nz - 1);
    g.iso = iso;
    return MR_OK;
}

static dim3 mc_grid(const McArgs& g) { return dim3((unsigned)g.kchunks, (unsigned)(g.ny - 1), (unsigned)(g.nx - 1)); }

}  // namespace mr

extern "C" int64_t mr_mc_blocks(int32_t nx, int32_t ny, int32_t nz) {
    if (nx < 2 || ny < 2 || nz < 2) return 0;
    return (int64_t)(nx - 1) * (ny - 1) * ((nz - 1 + mr::MC_THREADS - 1) / mr::MC_THREADS);
}

extern "C" int mr_mc_table(int8_t* table_host) {
    if (!table_host) return MR_ERR_INVALID;
    std::call_once(mr::g_table_once, [] { mr::build_table(mr::g_tri, mr::g_edge); });
    for (int m = 0; m < 256; ++m)
        for (int i = 0; i < 16; ++i) table_host[16 * m + i] = mr::g_tri[m][i];
    return MR_OK;
}

extern "C" int mr_mc_count(const float* vol, int32_t nx, int32_t ny, int32_t nz, float iso, int32_t* block_counts,
                           void* stream) {
    mr::McArgs g{};
    int rc = mr::fill_args(g, vol, nx, ny, nz, iso);
    if (rc != MR_OK) return rc;
    if (!block_counts) return MR_ERR_INVALID;
    rc = mr::ensure_table();
    if (rc != MR_OK) return rc;
    mr::mc_count_kernel<<<mr::mc_grid(g), mr::MC_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(g, block_counts);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

extern "C" int mr_mc_emit(const float* vol, int32_t nx, int32_t ny, int32_t nz, float iso, const double* origin,
                          double spacing, const int64_t* block_offsets, int64_t n_tri, int64_t* tri_edges,
                          float* tri_pos, void* stream) {
    mr::McArgs g{};
    int rc = mr::fill_args(g, vol, nx, ny, nz, iso);
    if (rc != MR_OK) return rc;
    if (!origin || !block_offsets || n_tri < 0 || (n_tri > 0 && (!tri_edges || !tri_pos))) return MR_ERR_INVALID;
    rc = mr::ensure_table();
    if (rc != MR_OK) return rc;
    if (n_tri == 0) return MR_OK;
    g.ox = (float)origin[0];
    g.oy = (float)origin[1];
    g.oz = (float)origin[2];
    g.h = (float)spacing;
    mr::mc_emit_kernel<<<mr::mc_grid(g), mr::MC_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        g, reinterpret_cast<const long long*>(block_offsets), (long long)n_tri,
        reinterpret_cast<long long*>(tri_edges), tri_pos);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}
