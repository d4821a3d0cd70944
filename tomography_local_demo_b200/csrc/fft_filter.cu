// Ingest + FDK/FBP row filter with register-resident FFTs (N = 32 ... 8192).
//
// Same contract as filter.cu (minirecast recon.py:34-104, flexray.py / hdf5.py raw
// correction); the FFT is organised for the SM instead of pass-by-pass in shared memory:
//   * one FFT (two detector rows packed as z = x1 + i x2; H is real and even, so the
//     filtered rows come back as Re and Im) is owned by G = N/32 threads, each holding
//     32 complex values in registers;
//   * N = 32 x R2 [x R3] mixed-radix Stockham: every pass is a radix-32 / R2 / R3 DFT
//     entirely in registers (compile-time twiddles), passes exchange through a padded
//     shared buffer (one float2 of padding per 32 keeps the transposes bank-conflict
//     free), synchronised per warp when G <= 32;
//   * the first pass reads its inputs straight from global memory (correction, -log and
//     FDK weight applied on the fly; the upper half of the zero-padded row is known to be
//     zero and its butterflies are pruned), and the last pass of the inverse transform
//     writes straight to the ring;
//   * the forward transform leaves X[n] in the registers of thread n mod G, which is
//     exactly the input layout of the inverse (forward FFT of conj(H X)), so the spectrum
//     never goes back to shared memory.
#include "mr_common.cuh"

namespace mr {
namespace fft {

constexpr double kPi = 3.14159265358979323846;

// Taylor series (|x| <= pi after reduction), evaluated at compile time for twiddles.
constexpr double csin_red(double x) {
    double term = x, sum = x;
    for (int n = 1; n < 24; ++n) {
        term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
        sum += term;
    }
    return sum;
}
constexpr double ccos_red(double x) {
    double term = 1.0, sum = 1.0;
    for (int n = 1; n < 24; ++n) {
        term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
        sum += term;
    }
    return sum;
}
constexpr double reduce(double x) {  // to (-pi, pi]
    while (x > kPi) x -= 2.0 * kPi;
    while (x <= -kPi) x += 2.0 * kPi;
    return x;
}

// W_R^k = exp(-2 pi i k / R) for k < R/2.
template <int R>
struct Twiddles {
    float re[R / 2 > 0 ? R / 2 : 1];
    float im[R / 2 > 0 ? R / 2 : 1];
    constexpr Twiddles() : re(), im() {
        for (int k = 0; k < R / 2; ++k) {
            const double a = reduce(-2.0 * kPi * k / R);
            re[k] = (float)ccos_red(a);
            im[k] = (float)csin_red(a);
        }
    }
};
template <int R>
__device__ constexpr Twiddles<R> kTw{};

template <int R, int K>
__device__ __forceinline__ float2 twiddle(float2 x) {
    if constexpr (K == 0) {
        return x;
    } else if constexpr (4 * K == R) {          // W = -i
        return make_float2(x.y, -x.x);
    } else {
        constexpr float c = kTw<R>.re[K], s = kTw<R>.im[K];
        // (x.x c - x.y s, x.x s + x.y c) as two packed operations (same roundings)
        return __ffma2_rn(make_float2(x.x, x.x), make_float2(c, s),
                          __fmul2_rn(make_float2(x.y, x.y), make_float2(-s, c)));
    }
}

// Radix-2 decimation-in-frequency DFT of R values v[OFF + S*m], m < R, in place; the
// result X[q] sits at v[OFF + S*bitrev(q)]. ZH: the upper half of the input is zero.
template <int R, int OFF, int S, bool ZH, int K = 0>
__device__ __forceinline__ void dif_stage(float2* v) {
    if constexpr (K < R / 2) {
        const float2 a = v[OFF + S * K];
        if constexpr (ZH) {
            v[OFF + S * (K + R / 2)] = twiddle<R, K>(a);
        } else {
            const float2 b = v[OFF + S * (K + R / 2)];
            v[OFF + S * K] = cadd(a, b);
            v[OFF + S * (K + R / 2)] = twiddle<R, K>(csub(a, b));
        }
        dif_stage<R, OFF, S, ZH, K + 1>(v);
    }
}
template <int R, int OFF, int S, bool ZH = false>
__device__ __forceinline__ void dif(float2* v) {
    if constexpr (R > 1) {
        dif_stage<R, OFF, S, ZH>(v);
        dif<R / 2, OFF, S>(v);
        dif<R / 2, OFF + S * (R / 2), S>(v);
    }
}

__host__ __device__ constexpr int bitrev(int x, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((x >> b) & 1) << (bits - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x / 2); }
__device__ __forceinline__ int pad(int a) { return a + (a >> 5); }

template <int LOG2N>
struct Plan {
    static constexpr int N = 1 << LOG2N;
    static constexpr int G = N / 32;                                   // threads per FFT
    static constexpr int R2 = N >= 1024 ? 32 : N / 32;                 // 1 -> single pass
    static constexpr int R3 = N / (32 * R2);                           // 1 -> no third pass
    static constexpr int FPB = 256 / G;                                // FFTs per block
    static constexpr int BUF = N + N / 32;                             // padded float2 per FFT
};

// Synchronises the G threads of one FFT (blocks of 256 threads, groups of whole warps):
// a warp barrier up to 32 threads, a named barrier per group (ids 1 .. 256 / G; 0 is
// __syncthreads) when several groups share the block, so one group's passes do not wait
// for the other groups' shared-memory transposes.
template <int G>
__device__ __forceinline__ void fft_sync() {
    static_assert(G % 32 == 0 || G < 32, "groups are whole warps");
    if constexpr (G <= 32) {
        __syncwarp();
    } else if constexpr (G < 256) {
        static_assert(256 / G <= 15, "named barrier ids 1..15");
        asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / G)), "n"(G) : "memory");
    } else {
        __syncthreads();
    }
}

// Forward FFT of the 32 values v[r] = x[j + G r] of the thread's FFT; on return
// v[idx] = X[j + G idx]. ZH: x[n] = 0 for n >= N/2.
template <int LOG2N, bool ZH>
__device__ __forceinline__ void fft32xN(float2 (&v)[32], float2* buf, const float2* __restrict__ T,
                                        const float2* __restrict__ twN, int j) {
    using P = Plan<LOG2N>;
    constexpr int N = P::N, G = P::G, R2 = P::R2, R3 = P::R3;
    // ---- pass 1: radix 32 (Ns = 1)
    dif<32, 0, 1, ZH>(v);
    if constexpr (R2 == 1) {               // N == 32: done, undo the bit reversal
        float2 t[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) t[q] = v[bitrev(q, 5)];
#pragma unroll
        for (int q = 0; q < 32; ++q) v[q] = t[q];
        return;
    } else {
        fft_sync<G>();                      // previous readers of buf are done
#pragma unroll
        for (int q = 0; q < 32; ++q) buf[pad(32 * j + q)] = v[bitrev(q, 5)];
        fft_sync<G>();
        // ---- pass 2: radix R2 (Ns = 32), 32/R2 butterflies per thread
        constexpr int NB2 = 32 / R2;
        constexpr int L2 = ilog2(R2);
#pragma unroll
        for (int b = 0; b < NB2; ++b) {
            const int jj = j + G * b;
            const int k = jj & 31;
#pragma unroll
            for (int r = 0; r < R2; ++r) {
                float2 x = buf[pad(jj + (N / R2) * r)];
                if (r > 0) x = cmul(x, T[(r * (32 / R2)) * 32 + k]);
                v[b * R2 + r] = x;
            }
        }
#pragma unroll
        for (int b = 0; b < NB2; ++b) {
            if constexpr (R2 == 32) dif<32, 0, 1>(v);
            else dif<R2, 0, 1>(v + b * R2);
        }
        if constexpr (R3 == 1) {
            // outputs X[(jj/32)*32*R2 + k + 32 m] with jj < 32 -> n = jj + 32 m = j + G (b + NB2 m)
            float2 t[32];
#pragma unroll
            for (int b = 0; b < NB2; ++b)
#pragma unroll
                for (int m = 0; m < R2; ++m) t[b + NB2 * m] = v[b * R2 + bitrev(m, L2)];
#pragma unroll
            for (int q = 0; q < 32; ++q) v[q] = t[q];
            return;
        } else {
            fft_sync<G>();
#pragma unroll
            for (int m = 0; m < 32; ++m) {          // NB2 == 1, jj = j
                const int k = j & 31;
                buf[pad((j >> 5) * 1024 + k + 32 * m)] = v[bitrev(m, 5)];
            }
            fft_sync<G>();
            // ---- pass 3: radix R3 (Ns = 1024), 32/R3 butterflies per thread
            constexpr int NB3 = 32 / R3;
            constexpr int L3 = ilog2(R3);
#pragma unroll
            for (int b = 0; b < NB3; ++b) {
                const int jj = j + G * b;          // < 1024
#pragma unroll
                for (int r = 0; r < R3; ++r) {
                    float2 x = buf[pad(jj + (N / R3) * r)];
                    if (r > 0) x = cmul(x, __ldg(twN + r * jj));
                    v[b * R3 + r] = x;
                }
            }
#pragma unroll
            for (int b = 0; b < NB3; ++b) dif<R3, 0, 1>(v + b * R3);
            float2 t[32];
#pragma unroll
            for (int b = 0; b < NB3; ++b)
#pragma unroll
                for (int m = 0; m < R3; ++m) t[b + NB3 * m] = v[b * R3 + bitrev(m, L3)];
#pragma unroll
            for (int q = 0; q < 32; ++q) v[q] = t[q];
        }
    }
}

// x W_32^K for any K < 32 (W_32^(K + 16) = -W_32^K), compile-time constants.
template <int K>
__device__ __forceinline__ float2 tw32(float2 x) {
    if constexpr (K >= 16) {
        const float2 y = twiddle<32, K - 16>(x);
        return make_float2(-y.x, -y.y);
    } else {
        return twiddle<32, K>(x);
    }
}
// v[b R3 + r] *= W_N^(r j) W_32^(r b) for r > 0, b < 32 / R3 (wj[r] = W_N^(r j)).
template <int R3, int B = 0, int RR = 1>
__device__ __forceinline__ void tw3_apply(float2 (&v)[32], const float2 (&wj)[R3]) {
    if constexpr (B < 32 / R3) {
        if constexpr (RR < R3) {
            v[B * R3 + RR] = tw32<(RR * B) % 32>(cmul(v[B * R3 + RR], wj[RR]));
            tw3_apply<R3, B, RR + 1>(v, wj);
        } else {
            tw3_apply<R3, B + 1, 1>(v, wj);
        }
    }
}

// N >= 1024: passes 1 and 2 are both radix 32; they share one copy of the DIF code in a
// runtime loop (straight-line radix-32 code is ~7 KB of SASS; four inlined copies
// thrash the instruction cache). Same input/output contract as fft32xN.
// SPLIT: the FFT's exchange buffer holds N + N/32 floats instead of float2s, and each
// transpose moves the real parts, then the imaginary parts (two more barriers, the same
// values in the same registers): half the shared memory, so that the row pair's dark /
// gain rows fit beside two CTAs an SM at 2048 and 4096 points.
template <int LOG2N, bool SPLIT = false>
__device__ __forceinline__ void fft_compact(float2 (&v)[32], float2* buf, const float2* __restrict__ T,
                                            const float2* __restrict__ twN, int j) {
    using P = Plan<LOG2N>;
    constexpr int N = P::N, G = P::G, R3 = P::R3;
    static_assert(P::R2 == 32, "compact path needs N >= 1024");
    const int k = j & 31;
    float* bf = reinterpret_cast<float*>(buf);
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            fft_sync<G>();
            if constexpr (SPLIT) {
                // real parts were stored at the end of pass 0; the imaginary parts of the
                // pass-0 results are still in v[].y
#pragma unroll
                for (int r = 0; r < 32; ++r) v[r].x = bf[pad(j + (N / 32) * r)];
                fft_sync<G>();
#pragma unroll
                for (int q = 0; q < 32; ++q) bf[pad(32 * j + q)] = v[bitrev(q, 5)].y;
                fft_sync<G>();
#pragma unroll
                for (int r = 0; r < 32; ++r) v[r].y = bf[pad(j + (N / 32) * r)];
#pragma unroll
                for (int r = 1; r < 32; ++r) v[r] = cmul(v[r], T[r * 32 + k]);
            } else {
#pragma unroll
                for (int r = 0; r < 32; ++r) {
                    float2 x = buf[pad(j + (N / 32) * r)];
                    if (r > 0) x = cmul(x, T[r * 32 + k]);
                    v[r] = x;
                }
            }
        }
        dif<32, 0, 1>(v);
        if (pass == 0) {
            fft_sync<G>();
            if constexpr (SPLIT) {
#pragma unroll
                for (int q = 0; q < 32; ++q) bf[pad(32 * j + q)] = v[bitrev(q, 5)].x;
            } else {
#pragma unroll
                for (int q = 0; q < 32; ++q) buf[pad(32 * j + q)] = v[bitrev(q, 5)];
            }
        }
    }
    if constexpr (R3 == 1) {
        float2 t[32];
#pragma unroll
        for (int m = 0; m < 32; ++m) t[m] = v[bitrev(m, 5)];
#pragma unroll
        for (int m = 0; m < 32; ++m) v[m] = t[m];
    } else {
        constexpr int NB3 = 32 / R3;
        constexpr int L3 = ilog2(R3);
        // SPLIT: W_N^(r (j + G b)) = W_N^(r j) W_32^(r b) (N = 32 G): R3 - 1 table reads a
        // thread instead of one per value, and a compile-time rotation
        float2 wj[R3];
        if constexpr (SPLIT) {
#pragma unroll
            for (int r = 1; r < R3; ++r) wj[r] = __ldg(twN + r * j);
        }
        fft_sync<G>();
        if constexpr (SPLIT) {
#pragma unroll
            for (int m = 0; m < 32; ++m) bf[pad((j >> 5) * 1024 + k + 32 * m)] = v[bitrev(m, 5)].x;
            fft_sync<G>();
#pragma unroll
            for (int b = 0; b < NB3; ++b)
#pragma unroll
                for (int r = 0; r < R3; ++r) v[b * R3 + r].x = bf[pad(j + G * b + (N / R3) * r)];
            fft_sync<G>();
#pragma unroll
            for (int m = 0; m < 32; ++m) bf[pad((j >> 5) * 1024 + k + 32 * m)] = v[bitrev(m, 5)].y;
            fft_sync<G>();
#pragma unroll
            for (int b = 0; b < NB3; ++b) {
                const int jj = j + G * b;
#pragma unroll
                for (int r = 0; r < R3; ++r) v[b * R3 + r].y = bf[pad(jj + (N / R3) * r)];
            }
            tw3_apply<R3>(v, wj);
        } else {
#pragma unroll
            for (int m = 0; m < 32; ++m) buf[pad((j >> 5) * 1024 + k + 32 * m)] = v[bitrev(m, 5)];
            fft_sync<G>();
#pragma unroll
            for (int b = 0; b < NB3; ++b) {
                const int jj = j + G * b;
#pragma unroll
                for (int r = 0; r < R3; ++r) {
                    float2 x = buf[pad(jj + (N / R3) * r)];
                    if (r > 0) x = cmul(x, __ldg(twN + r * jj));
                    v[b * R3 + r] = x;
                }
            }
        }
#pragma unroll
        for (int b = 0; b < NB3; ++b) dif<R3, 0, 1>(v + b * R3);
        float2 t[32];
#pragma unroll
        for (int b = 0; b < NB3; ++b)
#pragma unroll
            for (int m = 0; m < R3; ++m) t[b + NB3 * m] = v[b * R3 + bitrev(m, L3)];
#pragma unroll
        for (int q = 0; q < 32; ++q) v[q] = t[q];
    }
}

template <int LOG2N, bool SPLIT = false>
__device__ __forceinline__ void fft_any(float2 (&v)[32], float2* buf, const float2* __restrict__ T,
                                        const float2* __restrict__ twN, int j) {
    static_assert(!SPLIT || LOG2N >= 10, "split exchanges only on the compact path");
    if constexpr (LOG2N >= 10) fft_compact<LOG2N, SPLIT>(v, buf, T, twN, j);
    else fft32xN<LOG2N, false>(v, buf, T, twN, j);
}

}  // namespace fft

struct Filter2Args {
    const float* block;
    const uint16_t* raw;
    long long s_view, s_row;
    int bin, flip;
    const float* dark;
    const float* gain;
    const mr_filter_view* views;
    const float* H;
    const float2* tw;            // W_N^m, m < N
    void* ring;
    int dtype, rows, cols, pitch;
    long long slot_stride;
    int k;                       // views
};

template <bool RAW>
__device__ __forceinline__ float ingest_x(const Filter2Args& A, int v, int r, int c) {
    if (!RAW) return __ldg(A.block + (long long)v * A.s_view + (long long)r * A.s_row + c);
    const int b = A.bin;
    const int rr = A.flip ? (A.rows - 1 - r) : r;
    const uint16_t* p = A.raw + (long long)v * A.s_view + (long long)rr * b * A.s_row + (long long)c * b;
    float s;
    if (b == 1) {
        s = (float)__ldg(p);
    } else {
        s = 0.f;
        for (int dy = 0; dy < b; ++dy)
            for (int dx = 0; dx < b; ++dx) s += (float)__ldg(p + (long long)dy * A.s_row + dx);
        s = __fdiv_rn(s, (float)(b * b));
    }
    const int pix = r * A.cols + c;
    const float t = (s - __ldg(A.dark + pix)) * __ldg(A.gain + pix);
    return -__logf(fmaxf(t, 1e-3f));
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// FP32 value -> ring element (round to nearest for the 16-bit rings)
__device__ __forceinline__ float ring_cvt(const float*, float y) { return y; }
__device__ __forceinline__ __nv_bfloat16 ring_cvt(const __nv_bfloat16*, float y) { return __float2bfloat16_rn(y); }
__device__ __forceinline__ __half ring_cvt(const __half*, float y) { return __float2half_rn(y); }

// PREF: the next item's two input rows are copied to shared memory with cp.async while the
// current item's FFTs run (bin 1 only; rows of 4-byte aligned, 4-byte multiple length).
// SMF: the CTA's dark / gain rows sit in shared memory (every CTA works on one row pair).
// SPLIT: float exchange buffers (fft_compact), which leave room for those rows at N >= 2048.
template <int LOG2N, bool RAW, bool PREF, bool SMF, bool SPLIT = false>
__global__ void __launch_bounds__(256, 2) fft_filter_kernel(Filter2Args A, int split) {
    static_assert(!SPLIT || (RAW && PREF && SMF), "split exchanges come with the pair's fields");
    using P = fft::Plan<LOG2N>;
    constexpr int N = P::N, G = P::G, FPB = P::FPB;
    constexpr int ES = RAW ? 2 : 4;                      // input element size
    extern __shared__ float2 sm2[];
    float2* T = sm2;                                  // 32 x 32: T[a*32+k] = W_1024^(a k)
    const int f = threadIdx.x / G;
    const int j = threadIdx.x % G;
    constexpr int BUF_ES = SPLIT ? 4 : 8;               // bytes per exchange-buffer element
    unsigned char* bufs = reinterpret_cast<unsigned char*>(sm2 + 1024);
    float2* buf = reinterpret_cast<float2*>(bufs + (size_t)f * P::BUF * BUF_ES);
    const int row_bytes = ((A.cols * ES + 15) / 16) * 16;
    unsigned char* pref = bufs + (size_t)FPB * P::BUF * BUF_ES + f * 2 * row_bytes;

    if constexpr (P::R2 > 1) {
        // W_1024^(a k) = W_N^(a k N / 1024); for N < 1024 only a multiple of 1024/N is used
        for (int e = threadIdx.x; e < 1024; e += 256) {
            const int a = e >> 5, k = e & 31;
            const long long num = (long long)a * k * N;
            T[e] = (num % 1024 == 0) ? __ldg(A.tw + (int)((num / 1024) % N)) : make_float2(0.f, 0.f);
        }
    }
    __syncthreads();

    const int R = A.rows, C = A.cols;
    // item = pair * k + view. SMF: CTA b filters row pair b / split, views (b % split) * FPB
    // + f + m * split * FPB of it, so all its FFT slots share the pair's dark / gain rows,
    // held in shared memory. Otherwise the CTAs stride over all items (FPB consecutive
    // views of one pair at a time, the dark / gain rows shared through L1), which keeps
    // every SM busy to the end when few CTAs fit.
    const int pair = SMF ? (int)(blockIdx.x / split) : 0;
    const long long n_items = (long long)A.k * ((R + 1) / 2);
    float* fld = reinterpret_cast<float*>(pref - f * 2 * row_bytes + FPB * 2 * row_bytes);   // [4][C]
    float* wtab = fld + 4 * C;                     // [2][C] FDK weights of the CTA's first view
    float* wkey = wtab + 2 * C;                    // that view's a0, da, b0, db, sdd
    // SPLIT: H[0 .. N/2] (the spectrum is even, H[n] = H[N - n] bit for bit) after the key
    float* hs = wkey + 8;
    if constexpr (SPLIT) {
        for (int e = threadIdx.x; e <= N / 2; e += blockDim.x) hs[e] = __ldg(A.H + e);
    }
    if (RAW && SMF) {
        // dark of rows 2 pair, 2 pair + 1, then gain of the same rows
        // one float4 a column: dark of rows 2 pair, 2 pair + 1, gain of the same rows
        for (int e = threadIdx.x; e < 4 * C; e += blockDim.x) {
            const int q = e & 3, c = e >> 2;
            const int r = 2 * pair + (q & 1);
            fld[e] = r < R ? __ldg(((q >> 1) ? A.gain : A.dark) + (long long)r * C + c) : 0.f;
        }
        // the cosine weights of the pair's rows for the constants of the CTA's first view:
        // the views of one orbit usually share them, and a view that does reads its
        // weights here instead of computing them (the same operations, the same values)
        const int v0 = min((int)(blockIdx.x % split) * FPB, A.k - 1);
        const mr_filter_view f0 = A.views[v0];
        for (int e = threadIdx.x; e < 2 * C; e += blockDim.x) {      // one float2 a column
            const int q = e & 1, c = e >> 1;
            float w = 1.f;
            if (f0.sdd != 0.f) {
                const float aa = fmaf((float)c, f0.da, f0.a0);
                const float b1 = fmaf((float)(2 * pair), f0.db, f0.b0);
                const float b = q ? b1 + f0.db : b1;
                const float s2 = fmaf(f0.sdd, f0.sdd, aa * aa);
                w = f0.sdd * rsqrtf(fmaf(b, b, s2));
            }
            wtab[e] = w;
        }
        if (threadIdx.x == 0) {
            wkey[0] = f0.a0;
            wkey[1] = f0.da;
            wkey[2] = f0.b0;
            wkey[3] = f0.db;
            wkey[4] = f0.sdd;
        }
        __syncthreads();
    }
    // item = pair * k + view
    auto src_row = [&](long long item, int row) -> const unsigned char* {
        const int pr = (int)(item / A.k);
        const int v = (int)(item - (long long)pr * A.k);
        const int r = 2 * pr + row;
        if (RAW) {
            const int rr = A.flip ? (A.rows - 1 - r) : r;
            return reinterpret_cast<const unsigned char*>(A.raw + (long long)v * A.s_view + (long long)rr * A.s_row);
        }
        return reinterpret_cast<const unsigned char*>(A.block + (long long)v * A.s_view + (long long)r * A.s_row);
    };
    auto prefetch = [&](long long item) {
        if (PREF && item < n_items) {
            const int units = C * ES / 4;
            const int pr = (int)(item / A.k);
            const int nrow = (2 * pr + 1 < R) ? 2 : 1;
            for (int row = 0; row < nrow; ++row) {
                const unsigned char* src = src_row(item, row);
                for (int u = j; u < units; u += G) cp_async4(pref + row * row_bytes + 4 * u, src + 4 * u);
            }
        }
        if (PREF) cp_async_commit();
    };
    const long long start = SMF ? (long long)pair * A.k + (long long)(blockIdx.x % split) * FPB
                                : (long long)blockIdx.x * FPB;
    const long long end = SMF ? (long long)(pair + 1) * A.k : n_items;
    const long long step = SMF ? (long long)split * FPB : (long long)gridDim.x * FPB;
    if (start + f < end) prefetch(start + f);
    else if (PREF) cp_async_commit();
    for (long long base = start; base < end; base += step) {
        const long long item = base + f;
        const bool live = item < end;                  // uniform per FFT group
        const int pr = SMF ? pair : (live ? (int)(item / A.k) : 0);
        const int v = live ? (int)(item - (long long)pr * A.k) : 0;
        const int r1 = 2 * pr;
        const mr_filter_view fv = A.views[v];
        if (PREF) {
            cp_async_wait_all();
            fft::fft_sync<G>();                         // the staged rows are visible to the group
        }
        float2 x[32];
        const bool tab = RAW && SMF && fv.a0 == wkey[0] && fv.da == wkey[1] && fv.b0 == wkey[2] &&
                         fv.db == wkey[3] && fv.sdd == wkey[4];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int c = j + G * q;
            float a = 0.f, b = 0.f;
            if (live && c < C) {
                float w1 = 1.f, w2 = 1.f;
                if (tab) {
                    const float2 w = reinterpret_cast<const float2*>(wtab)[c];
                    w1 = w.x;
                    w2 = w.y;
                } else if (fv.sdd != 0.f) {
                    const float aa = fmaf((float)c, fv.da, fv.a0);
                    const float b1 = fmaf((float)r1, fv.db, fv.b0), b2 = b1 + fv.db;
                    const float s2 = fmaf(fv.sdd, fv.sdd, aa * aa);
                    w1 = fv.sdd * rsqrtf(fmaf(b1, b1, s2));
                    w2 = fv.sdd * rsqrtf(fmaf(b2, b2, s2));
                }
                if (PREF) {
                    float x1, x2 = 0.f;
                    if (RAW) {
                        const int pix = r1 * A.cols + c;
                        const float s1 = (float)reinterpret_cast<const uint16_t*>(pref)[c];
                        float4 dg = make_float4(0.f, 0.f, 0.f, 0.f);      // dark 1, dark 2, gain 1, gain 2
                        if (SMF) {
                            dg = reinterpret_cast<const float4*>(fld)[c];
                        } else {
                            dg.x = __ldg(A.dark + pix);
                            dg.z = __ldg(A.gain + pix);
                        }
                        x1 = -__logf(fmaxf((s1 - dg.x) * dg.z, 1e-3f));
                        if (r1 + 1 < R) {
                            const float s2r = (float)reinterpret_cast<const uint16_t*>(pref + row_bytes)[c];
                            if (!SMF) {
                                dg.y = __ldg(A.dark + pix + A.cols);
                                dg.w = __ldg(A.gain + pix + A.cols);
                            }
                            x2 = -__logf(fmaxf((s2r - dg.y) * dg.w, 1e-3f));
                        }
                    } else {
                        x1 = reinterpret_cast<const float*>(pref)[c];
                        if (r1 + 1 < R) x2 = reinterpret_cast<const float*>(pref + row_bytes)[c];
                    }
                    a = x1 * w1;
                    b = x2 * w2;
                } else {
                    a = ingest_x<RAW>(A, v, r1, c) * w1;
                    if (r1 + 1 < R) b = ingest_x<RAW>(A, v, r1 + 1, c) * w2;
                }
            }
            x[q] = make_float2(a, b);
        }
        if (PREF) {
            fft::fft_sync<G>();                         // everyone has read the staged rows
            if (item + step < end) prefetch(item + step);
            else cp_async_commit();
        }
#pragma unroll
        for (int q = 16; q < 32; ++q) x[q] = make_float2(0.f, 0.f);
        const float g = fv.gain * fv.out_scale;
        // forward FFT, conj(H X), forward FFT again (= N * conj of the inverse): one call site,
        // except at 1024 points, where two copies let the output permutation of the first
        // transform stay a renaming of registers
        constexpr int IT_UNROLL = LOG2N == 10 ? 2 : 1;
#pragma unroll (IT_UNROLL)
        for (int it = 0; it < 2; ++it) {
            fft::fft_any<LOG2N, SPLIT>(x, buf, T, A.tw, j);
            if (it == 0) {
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    // n = j + G q is below N/2 exactly when q < 16
                    const float hn = SPLIT ? (q < 16 ? hs[j + G * q] : hs[N - j - G * q]) : __ldg(A.H + j + G * q);
                    const float h = hn * g;
                    x[q] = __fmul2_rn(x[q], make_float2(h, -h));
                }
            }
        }
        if (live) {
            const long long o1 = (long long)fv.slot * A.slot_stride + (long long)r1 * A.pitch;
            const bool two = r1 + 1 < R;
            // one store loop per ring type (no per-column type dispatch). Columns c = j + G q:
            // q < 16 covers c < N/2, which holds the row's C columns (the entry points
            // require N >= 2 C) and, for the rings the host builds, the whole pitch; the
            // columns of a wider pitch (up to N) are padding and get zeros in the second loop
            auto put = [&](auto* ring) {
                auto* o = ring + o1;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int c = j + G * q;
                    if (c < A.pitch) {
                        o[c] = ring_cvt(o, c < C ? x[q].x : 0.f);
                        if (two) o[c + A.pitch] = ring_cvt(o, c < C ? -x[q].y : 0.f);
                    }
                }
                for (int c = N / 2 + j; c < min(A.pitch, N); c += G) {
                    o[c] = ring_cvt(o, 0.f);
                    if (two) o[c + A.pitch] = ring_cvt(o, 0.f);
                }
            };
            if (A.dtype == MR_F32) put(static_cast<float*>(A.ring));
            else if (A.dtype == MR_BF16) put(static_cast<__nv_bfloat16*>(A.ring));
            else put(static_cast<__half*>(A.ring));
        }
    }
}

template <int LOG2N, bool RAW>
static int launch_fft_filter(const Filter2Args& A, cudaStream_t st) {
    using P = fft::Plan<LOG2N>;
    constexpr int ES = RAW ? 2 : 4;
    const size_t base_smem = (1024 + (size_t)P::FPB * P::BUF) * sizeof(float2);
    const size_t split_smem = 1024 * sizeof(float2) + (size_t)P::FPB * P::BUF * sizeof(float);
    const size_t row_bytes = ((size_t)A.cols * ES + 15) / 16 * 16;
    const size_t pref_smem = (size_t)P::FPB * 2 * row_bytes;
    // staged input rows need bin 1 and 4-byte aligned rows of a 4-byte multiple length
    const long long elem_align = 4 / ES;
    const bool pref = A.bin == 1 && (A.cols * ES) % 4 == 0 && A.s_view % elem_align == 0 &&
                      A.s_row % elem_align == 0 &&
                      (reinterpret_cast<uintptr_t>(RAW ? (const void*)A.raw : (const void*)A.block) & 3) == 0 &&
                      base_smem + pref_smem <= 200 * 1024;
    // the dark / gain rows of the CTA's row pair in shared memory when two CTAs still fit an SM
    const size_t fld_smem = (size_t)6 * A.cols * sizeof(float) + 8 * sizeof(float);
    bool smf = RAW && pref && base_smem + pref_smem + fld_smem <= 112 * 1024;
    // 2048 / 4096 points: with float exchange buffers the fields (and half the spectrum)
    // fit beside two CTAs an SM
    const size_t hs_smem = (size_t)(P::N / 2 + 1) * sizeof(float);
    const bool split_smf = RAW && LOG2N >= 11 && LOG2N <= 12 && pref && !smf &&
                           split_smem + pref_smem + fld_smem + hs_smem <= 112 * 1024;
    smf = smf || split_smf;
    const size_t smem = (split_smf ? split_smem + hs_smem : base_smem) + (pref ? pref_smem : 0) +
                        (smf ? fld_smem : 0);
    auto kern = split_smf ? fft_filter_kernel<LOG2N, RAW, true, true, (RAW && LOG2N >= 11 && LOG2N <= 12)>
              : smf       ? fft_filter_kernel<LOG2N, RAW, true, true>
              : (pref ? fft_filter_kernel<LOG2N, RAW, true, false> : fft_filter_kernel<LOG2N, RAW, false, false>);
    MR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // SMF: one row pair per CTA, its views split over `split` CTAs of FPB FFT slots (about
    // eight views a slot); else a grid of two waves of eight CTAs per SM striding over all
    const long long pairs = (A.rows + 1) / 2;
    const long long split = (A.k + 8LL * P::FPB - 1) / (8LL * P::FPB);
    long long grid = pairs * split;
    if (!smf) {
        int dev = 0, sms = 148;
        MR_CUDA_TRY(cudaGetDevice(&dev));
        MR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const long long need = ((long long)A.k * pairs + P::FPB - 1) / P::FPB;
        grid = need < 2LL * sms * 8 ? need : 2LL * sms * 8;
    }
    if (A.k <= 0 || grid <= 0) return MR_OK;
    if (grid > 2147483647LL) return MR_ERR_UNSUPPORTED;
    kern<<<(unsigned)grid, 256, smem, st>>>(A, (int)split);
    MR_CUDA_TRY(cudaGetLastError());
    return MR_OK;
}

template <bool RAW>
int launch_fft_filter_any(const Filter2Args& A, int log2n, cudaStream_t st) {
    switch (log2n) {
        case 5: return launch_fft_filter<5, RAW>(A, st);
        case 6: return launch_fft_filter<6, RAW>(A, st);
        case 7: return launch_fft_filter<7, RAW>(A, st);
        case 8: return launch_fft_filter<8, RAW>(A, st);
        case 9: return launch_fft_filter<9, RAW>(A, st);
        case 10: return launch_fft_filter<10, RAW>(A, st);
        case 11: return launch_fft_filter<11, RAW>(A, st);
        case 12: return launch_fft_filter<12, RAW>(A, st);
        case 13: return launch_fft_filter<13, RAW>(A, st);
        default: return MR_ERR_UNSUPPORTED;
    }
}

template int launch_fft_filter_any<false>(const Filter2Args&, int, cudaStream_t);
template int launch_fft_filter_any<true>(const Filter2Args&, int, cudaStream_t);

}  // namespace mr
