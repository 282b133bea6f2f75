/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatements of the reference (iitd-plos/unicorn testSuite) algorithms
 * on the B200 subtask path.  They exist to CHECK the CUDA kernels: only
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py load
 * this library.  Nothing in unicorn_b200/ links or calls it.
 *
 * Parity is pinned two ways: (1) against the reference's own CPU callbacks
 * compiled from the reference sources into oracle/_ref (oracle/ref/Makefile),
 * on identical seeded inputs; (2) against the golden fixtures committed under
 * tests/golden/ (generated by tests/golden/make_golden.py from (1)).
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define ORC_MAX_FILTER_DIM 32

/* Number of worker threads the row-parallel oracles use (default 1). */
static int g_threads = 1;
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }

/* Run body(lo, hi, arg) over [0, n) split into g_threads contiguous chunks. */
typedef void (*orc_range_fn)(long lo, long hi, void* arg);
struct orc_job { orc_range_fn fn; void* arg; long lo, hi; };
static void* orc_thread_main(void* p) {
    struct orc_job* j = (struct orc_job*)p;
    j->fn(j->lo, j->hi, j->arg);
    return NULL;
}
static void orc_parallel_for(long n, orc_range_fn fn, void* arg) {
    int t = g_threads;
    if (t > n) t = (int)(n > 0 ? n : 1);
    if (t <= 1) { fn(0, n, arg); return; }
    pthread_t th[256];
    struct orc_job jobs[256];
    for (int k = 0; k < t; ++k) {
        jobs[k].fn = fn; jobs[k].arg = arg;
        jobs[k].lo = n * k / t; jobs[k].hi = n * (k + 1) / t;
        if (k > 0) pthread_create(&th[k], NULL, orc_thread_main, &jobs[k]);
    }
    orc_thread_main(&jobs[0]);
    for (int k = 1; k < t; ++k) pthread_join(th[k], NULL);
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/*
 * imageFilter over an output rectangle, NATURAL views of the whole image.
 * Follows imageFilter_cpu, testSuite/imageFiltering/source/code/src/
 * imageFiltering.cpp:419-468: taps clamp to the image border (:433-434), the
 * input address space holds image row m in buffer row H-1-m (:438), output
 * byte 0 of a pixel accumulates input byte 2 and byte 2 accumulates input
 * byte 0 (:457-467).  mode 0 (wrap): the accumulator is a char, so the result
 * is the exact sum reduced mod 256 (two's complement); mode 1 (clamp):
 * unsigned input bytes, exact int sum clamped to [0,255].
 */
struct imgf_args {
    const uint8_t* in; uint8_t* out; int W, H, R; const int8_t* filter; int mode, r0, c0, c1;
};

static void imgf_rows(long lo, long hi, void* p) {
    const struct imgf_args* a = (const struct imgf_args*)p;
    const int W = a->W, H = a->H, R = a->R;
    for (long ii = lo; ii < hi; ++ii) {
        const int i = a->r0 + (int)ii;
        for (int j = a->c0; j < a->c1; ++j) {
            int acc[3] = {0, 0, 0};
            for (int ky = 0; ky <= 2 * R; ++ky) {
                const int m = clampi(i - R + ky, 0, H - 1);
                const uint8_t* row = a->in + (size_t)(H - 1 - m) * 3 * W;
                for (int kx = 0; kx <= 2 * R; ++kx) {
                    const int n = clampi(j - R + kx, 0, W - 1);
                    const int f = a->filter[ky * ORC_MAX_FILTER_DIM + kx];
                    if (a->mode == 0) {
                        acc[0] += (int8_t)row[3 * n + 2] * f;
                        acc[1] += (int8_t)row[3 * n + 1] * f;
                        acc[2] += (int8_t)row[3 * n + 0] * f;
                    } else {
                        acc[0] += row[3 * n + 2] * f;
                        acc[1] += row[3 * n + 1] * f;
                        acc[2] += row[3 * n + 0] * f;
                    }
                }
            }
            uint8_t* o = a->out + ((size_t)i * W + j) * 3;
            for (int c = 0; c < 3; ++c)
                o[c] = a->mode == 0 ? (uint8_t)(acc[c] & 0xff) : (uint8_t)clampi(acc[c], 0, 255);
        }
    }
}

void orc_image_filter(const uint8_t* in, uint8_t* out, int W, int H, int R, const int8_t* filter,
                      int mode, int r0, int r1, int c0, int c1) {
    struct imgf_args a = {in, out, W, H, R, filter, mode, r0, c0, c1};
    orc_parallel_for(r1 - r0, imgf_rows, &a);
}

/*
 * Inclusive prefix sum, uint32 in -> uint64 out.  Follows serialPrefixSum,
 * testSuite/prefixSum/source/code/src/prefixSum.cpp:47-53 (out[0] = in[0];
 * out[i] = in[i] + out[i-1]) with the sum widened to 64 bits.
 */
void orc_prefix_sum_u32_u64(const uint32_t* in, uint64_t* out, size_t n) {
    if (n == 0) return;
    out[0] = in[0];
    for (size_t i = 1; i < n; ++i) out[i] = (uint64_t)in[i] + out[i - 1];
}

/*
 * One stable counting-sort round on the digit (key >> shift) & (2^bits - 1).
 * Follows serialRadixSortRound, testSuite/radixSort/source/code/src/
 * radixSort.cpp:55-69: count the bins, turn counts into inclusive positions,
 * then place keys walking the input backwards (which keeps equal digits in
 * input order).  `bins_out` (may be NULL) receives the per-digit counts, as the
 * reference hands them to its redistribution callback.
 */
void orc_radix_round_u32(const uint32_t* in, uint32_t* out, size_t n, int shift, int bits, uint32_t* bins_out) {
    const uint32_t nb = 1u << bits, mask = nb - 1;
    size_t* bins = (size_t*)calloc(nb, sizeof(size_t));
    for (size_t i = 0; i < n; ++i) ++bins[(in[i] >> shift) & mask];
    if (bins_out)
        for (uint32_t k = 0; k < nb; ++k) bins_out[k] = (uint32_t)bins[k];
    for (uint32_t k = 1; k < nb; ++k) bins[k] += bins[k - 1];
    for (size_t j = n; j-- > 0;) out[--bins[(in[j] >> shift) & mask]] = in[j];
    free(bins);
}

/*
 * Full LSD sort: rounds over digits [begin_bit, end_bit) of width `bits`,
 * ping-ponging through `tmp` (serialLsbRadixSort, radixSort.cpp:71-114).
 * The result is left in `keys`.
 */
void orc_radix_sort_u32(uint32_t* keys, uint32_t* tmp, size_t n, int begin_bit, int end_bit, int bits) {
    uint32_t* a = keys;
    uint32_t* b = tmp;
    for (int s = begin_bit; s < end_bit; s += bits) {
        orc_radix_round_u32(a, b, n, s, bits, NULL);
        uint32_t* t = a; a = b; b = t;
    }
    if (a != keys) memcpy(keys, a, n * sizeof(uint32_t));
}

/*
 * PageRank, FP64, pulled over CSR in-edges (row_ptr[N+1], col[E] = sources).
 * The formula of serialPageRank / pageRank_cpu (testSuite/pageRank/source/
 * code/src/pageRank.cpp:237-276, :336-378): r'[v] = sum over u->v of
 * d * r[u] / outdeg(u), no teleport term, pages without out-links give
 * nothing.  Everything is carried in double; `rank_init` is the fp32 initial
 * vector, `out` receives the ranks after `iters` iterations.
 */
struct pr_args {
    const uint32_t* row_ptr; const uint32_t* col; const double* contrib; double* next; long n;
};
static void pr_rows(long lo, long hi, void* p) {
    const struct pr_args* a = (const struct pr_args*)p;
    for (long v = lo; v < hi; ++v) {
        double s = 0.0;
        for (uint32_t e = a->row_ptr[v]; e < a->row_ptr[v + 1]; ++e) s += a->contrib[a->col[e]];
        a->next[v] = s;
    }
}
void orc_pagerank_f64(const uint32_t* row_ptr, const uint32_t* col, const uint32_t* outdeg, uint32_t n, int iters,
                      double damping, const float* rank_init, double* out) {
    double* r = (double*)malloc(sizeof(double) * n);
    double* c = (double*)malloc(sizeof(double) * n);
    for (uint32_t v = 0; v < n; ++v) r[v] = rank_init[v];
    for (int it = 0; it < iters; ++it) {
        for (uint32_t v = 0; v < n; ++v) c[v] = outdeg[v] ? damping * r[v] / (double)outdeg[v] : 0.0;
        struct pr_args a = {row_ptr, col, c, r, (long)n};
        orc_parallel_for(n, pr_rows, &a);
    }
    memcpy(out, r, sizeof(double) * n);
    free(r);
    free(c);
}

/*
 * PageRank in fp32 with the reference's push order: for each source page in
 * ascending order, incr = (0.85f * r[u]) / (float)outdeg(u) is added to every
 * target in edge order (pageRank.cpp:262-274 / :359-372).  `edge_src` must be
 * sorted by source (stable in generation order within a source).
 */
void orc_pagerank_push_f32(const uint32_t* edge_src, const uint32_t* edge_dst, uint64_t n_edges, uint32_t n,
                           const uint32_t* outdeg, int iters, float damping, const float* rank_init, float* out) {
    float* r = (float*)malloc(sizeof(float) * n);
    float* g = (float*)malloc(sizeof(float) * n);
    memcpy(r, rank_init, sizeof(float) * n);
    for (int it = 0; it < iters; ++it) {
        memset(g, 0, sizeof(float) * n);
        for (uint64_t e = 0; e < n_edges; ++e) {
            const uint32_t u = edge_src[e];
            const float incr = (float)(damping * r[u]) / (float)outdeg[u];
            g[edge_dst[e]] += incr;
        }
        float* t = r; r = g; g = t;
    }
    memcpy(out, r, sizeof(float) * n);
    free(r);
    free(g);
}

/*
 * Unpivoted Crout LU, column-major, in FP64.  Follows serialLUDecomposition,
 * testSuite/luDecomposition/source/code/src/luDecomposition.cpp:116-125: for
 * column i, the row to the right of the diagonal is scaled by 1/a_ii (cblas
 * scal with stride ld) and the trailing block gets the rank-1 update
 * a_rc -= a_ri * a_ic (cblas ger).  `a` (n x n, ld) is factored in place.
 */
void orc_lu_crout_f64(double* a, int n, long ld) {
    for (int i = 0; i < n - 1; ++i) {
        const double inv = 1.0 / a[i + (long)i * ld];
        for (int c = i + 1; c < n; ++c) a[i + (long)c * ld] *= inv;
        for (int c = i + 1; c < n; ++c) {
            const double u = a[i + (long)c * ld];
            double* col = a + (long)c * ld;
            const double* li = a + (long)i * ld;
            for (int r = i + 1; r < n; ++r) col[r] -= li[r] * u;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Subtask reduction: pmReducer::ReduceMemories                              */
/* (source/code/src/pmReducer.cpp:590-700) folds subtask 2's shadow memory   */
/* into subtask 1's element by element; bitwise operations on floats and     */
/* doubles act on the values converted to uint32 / uint64                    */
/* (pmReducer.cpp:408-423); LOGICAL_XOR is a != b.  op / type take the       */
/* pmReductionOpType / pmReductionDataType values.  Pinned bit for bit to   */
/* the reference's own ReduceMemories, cut unchanged out of pmReducer.cpp    */
/* into oracle/_ref/libref_reduce.so (tests/test_reduce_ref.py), and to its  */
/* golden outputs (tests/golden/reduce_golden.npz).                          */
/* ------------------------------------------------------------------------ */
#define ORC_FOLD(T, B)                                                                        \
    do {                                                                                      \
        T* x = (T*)a;                                                                         \
        const T* y = (const T*)b;                                                             \
        for (size_t i = 0; i < n; ++i) {                                                      \
            switch (op) {                                                                     \
                case 0: x[i] = x[i] + y[i]; break;                                            \
                case 1: x[i] = y[i] < x[i] ? y[i] : x[i]; break;                              \
                case 2: x[i] = x[i] < y[i] ? y[i] : x[i]; break;                              \
                case 3: x[i] = x[i] * y[i]; break;                                            \
                case 4: x[i] = (T)(x[i] && y[i]); break;                                      \
                case 5: x[i] = (T)((B)x[i] & (B)y[i]); break;                                 \
                case 6: x[i] = (T)(x[i] || y[i]); break;                                      \
                case 7: x[i] = (T)((B)x[i] | (B)y[i]); break;                                 \
                case 8: x[i] = (T)(x[i] != y[i]); break;                                      \
                default: x[i] = (T)((B)x[i] ^ (B)y[i]); break;                                \
            }                                                                                 \
        }                                                                                     \
    } while (0)

int orc_reduce_fold(int op, int type, void* a, const void* b, size_t n) {
    if (op < 0 || op > 9) return -1;
    switch (type) {
        case 0: ORC_FOLD(int32_t, int32_t); break;
        case 1: ORC_FOLD(uint32_t, uint32_t); break;
        case 2: ORC_FOLD(int64_t, int64_t); break;
        case 3: ORC_FOLD(uint64_t, uint64_t); break;
        case 4: ORC_FOLD(float, uint32_t); break;
        case 5: ORC_FOLD(double, uint64_t); break;
        default: return -1;
    }
    return 0;
}
