/*
 * TEST INFRASTRUCTURE ONLY - the CPU oracle of the back-projection path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it, as the
 * checker; the product never links, loads or calls it.
 *
 * A plain-C restatement of minirecast's Numba kernels, loop for loop:
 *   _bil_nb            recon.py:156-173  bilinear tap, zero outside [0,R)x[0,C)
 *   bp_parallel_numba  recon.py:175-191
 *   bp_cone_numba      recon.py:193-219
 * Accumulation is in float64 as in the reference (acc = 0.0, out = np.zeros(M)).
 * The q stack is float32 (the reference's store) or float64 (the FP64 oracle).
 * Parallel over output points with POSIX threads (static blocks), like Numba's prange.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <string.h>
#include <unistd.h>

static int g_threads = 0;   /* 0 = all online cores */

/* Set the thread count (n > 0; n <= 0 keeps it) and return the count in use. */
int oracle_threads(int n) {
    if (n > 0) g_threads = n;
    if (g_threads <= 0) {
        long c = sysconf(_SC_NPROCESSORS_ONLN);
        g_threads = c > 0 ? (int)c : 1;
    }
    return g_threads;
}

typedef struct {
    void (*body)(const void* args, long i0, long i1);
    const void* args;
    long i0, i1;
} span_t;

static void* span_main(void* p) {
    span_t* s = (span_t*)p;
    s->body(s->args, s->i0, s->i1);
    return NULL;
}

/* Run body over [0, M) split in equal static blocks across the threads. */
static void parallel_for(long M, void (*body)(const void*, long, long), const void* args) {
    int T = oracle_threads(0);
    if (T > 256) T = 256;
    if (M < 1024 || T == 1) { body(args, 0, M); return; }
    pthread_t th[256];
    span_t sp[256];
    int started[256];
    const long per = (M + T - 1) / T;
    for (int t = 0; t < T; ++t) {
        sp[t].body = body; sp[t].args = args;
        sp[t].i0 = t * per < M ? t * per : M;
        sp[t].i1 = (t + 1) * per < M ? (t + 1) * per : M;
        started[t] = pthread_create(&th[t], NULL, span_main, &sp[t]) == 0;
        if (!started[t]) body(args, sp[t].i0, sp[t].i1);
    }
    for (int t = 0; t < T; ++t)
        if (started[t]) pthread_join(th[t], NULL);
}

#define BIL_BODY(QT)                                                              \
    if (!(r > -1e9 && r < 1e9 && c > -1e9 && c < 1e9)) return 0.0;                \
    const long r0 = (long)floor(r), c0 = (long)floor(c);                          \
    const double fr = r - (double)r0, fc = c - (double)c0;                        \
    double v = 0.0;                                                               \
    const QT* im = img + k * R * C;                                               \
    if (0 <= r0 && r0 < R) {                                                      \
        if (0 <= c0 && c0 < C) v += (1.0 - fr) * (1.0 - fc) * (double)im[r0 * C + c0];       \
        if (0 <= c0 + 1 && c0 + 1 < C) v += (1.0 - fr) * fc * (double)im[r0 * C + c0 + 1];  \
    }                                                                             \
    if (0 <= r0 + 1 && r0 + 1 < R) {                                              \
        if (0 <= c0 && c0 < C) v += fr * (1.0 - fc) * (double)im[(r0 + 1) * C + c0];         \
        if (0 <= c0 + 1 && c0 + 1 < C) v += fr * fc * (double)im[(r0 + 1) * C + c0 + 1];     \
    }                                                                             \
    return v;

static inline double bil_f32(const float* img, long k, double r, double c, long R, long C) {
    BIL_BODY(float)
}
static inline double bil_f64(const double* img, long k, double r, double c, long R, long C) {
    BIL_BODY(double)
}

#define BP_CONE_BODY(BIL)                                                         \
    const double cr = (R - 1) / 2.0, cc = (C - 1) / 2.0;                          \
    for (long i = i_begin; i < i_end; ++i) {                                      \
        const double px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];   \
        double acc = 0.0;                                                         \
        for (long k = 0; k < A; ++k) {                                            \
            const double rx = px - S[3 * k], ry = py - S[3 * k + 1], rz = pz - S[3 * k + 2]; \
            const double L = rx * Nn[3 * k] + ry * Nn[3 * k + 1] + rz * Nn[3 * k + 2];       \
            const double t = SDD[k] / L;                                          \
            const double X0 = S[3 * k] + t * rx - D[3 * k];                       \
            const double X1 = S[3 * k + 1] + t * ry - D[3 * k + 1];               \
            const double X2 = S[3 * k + 2] + t * rz - D[3 * k + 2];               \
            const double col = X0 * UU[3 * k] + X1 * UU[3 * k + 1] + X2 * UU[3 * k + 2] + cc; \
            const double row = X0 * VV[3 * k] + X1 * VV[3 * k + 1] + X2 * VV[3 * k + 2] + cr; \
            const double w = SOD[k] / L;                                          \
            acc += w * w * BIL(q, k, row, col, R, C);                             \
        }                                                                         \
        out[i] = acc * scale;                                                     \
    }

#define BP_PAR_BODY(BIL)                                                          \
    const double cr = (R - 1) / 2.0, cc = (C - 1) / 2.0 + col_shift;              \
    for (long i = i_begin; i < i_end; ++i) {                                      \
        const double x = pts[3 * i], y = pts[3 * i + 1];                          \
        const double row = pts[3 * i + 2] / pv + cr;                              \
        double acc = 0.0;                                                         \
        for (long k = 0; k < A; ++k) {                                            \
            const double col = (-x * sin_t[k] + y * cos_t[k]) / pu + cc;          \
            acc += BIL(q, k, row, col, R, C);                                     \
        }                                                                         \
        out[i] = acc * scale;                                                     \
    }

typedef struct {
    const void* q; long A, R, C;
    const double *S, *D, *UU, *VV, *Nn, *SDD, *SOD, *pts;
    double scale; double* out;
} cone_args;

typedef struct {
    const void* q; long A, R, C;
    const double *cos_t, *sin_t; double pu, pv;
    const double* pts; double scale, col_shift; double* out;
} par_args;

#define UNPACK_CONE(QT)                                                           \
    const cone_args* a = (const cone_args*)vp;                                    \
    const QT* q = (const QT*)a->q;                                                \
    const long A = a->A, R = a->R, C = a->C;                                      \
    const double *S = a->S, *D = a->D, *UU = a->UU, *VV = a->VV, *Nn = a->Nn;     \
    const double *SDD = a->SDD, *SOD = a->SOD, *pts = a->pts;                     \
    const double scale = a->scale; double* out = a->out;

#define UNPACK_PAR(QT)                                                            \
    const par_args* a = (const par_args*)vp;                                      \
    const QT* q = (const QT*)a->q;                                                \
    const long A = a->A, R = a->R, C = a->C;                                      \
    const double *cos_t = a->cos_t, *sin_t = a->sin_t, pu = a->pu, pv = a->pv;    \
    const double* pts = a->pts; const double scale = a->scale, col_shift = a->col_shift; \
    double* out = a->out;

static void cone_f32_body(const void* vp, long i_begin, long i_end) { UNPACK_CONE(float) BP_CONE_BODY(bil_f32) }
static void cone_f64_body(const void* vp, long i_begin, long i_end) { UNPACK_CONE(double) BP_CONE_BODY(bil_f64) }
static void par_f32_body(const void* vp, long i_begin, long i_end) { UNPACK_PAR(float) BP_PAR_BODY(bil_f32) }
static void par_f64_body(const void* vp, long i_begin, long i_end) { UNPACK_PAR(double) BP_PAR_BODY(bil_f64) }

void oracle_bp_cone_f32(const float* q, long A, long R, long C, const double* S, const double* D,
                        const double* UU, const double* VV, const double* Nn, const double* SDD,
                        const double* SOD, const double* pts, long M, double scale, double* out) {
    cone_args a = {q, A, R, C, S, D, UU, VV, Nn, SDD, SOD, pts, scale, out};
    parallel_for(M, cone_f32_body, &a);
}

void oracle_bp_cone_f64(const double* q, long A, long R, long C, const double* S, const double* D,
                        const double* UU, const double* VV, const double* Nn, const double* SDD,
                        const double* SOD, const double* pts, long M, double scale, double* out) {
    cone_args a = {q, A, R, C, S, D, UU, VV, Nn, SDD, SOD, pts, scale, out};
    parallel_for(M, cone_f64_body, &a);
}

void oracle_bp_parallel_f32(const float* q, long A, long R, long C, const double* cos_t,
                            const double* sin_t, double pu, double pv, const double* pts, long M,
                            double scale, double col_shift, double* out) {
    par_args a = {q, A, R, C, cos_t, sin_t, pu, pv, pts, scale, col_shift, out};
    parallel_for(M, par_f32_body, &a);
}

void oracle_bp_parallel_f64(const double* q, long A, long R, long C, const double* cos_t,
                            const double* sin_t, double pu, double pv, const double* pts, long M,
                            double scale, double col_shift, double* out) {
    par_args a = {q, A, R, C, cos_t, sin_t, pu, pv, pts, scale, col_shift, out};
    parallel_for(M, par_f64_body, &a);
}
