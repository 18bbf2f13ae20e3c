/*
 * zoda_oracle.c -- CPU restatement of zoda-cu's column-wise Reed-Solomon
 * extension over BabyBear (p = 2^31 - 2^27 + 1).
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker: the tests, the
 * smoke check and the bench's CPU-baseline leg call it. The product (the CUDA
 * library under zoda-cu_b200/) never links, loads or calls it.
 *
 * The reference's CPU path is Rust (src/ntt/cpu.rs, src/field/babybear.rs,
 * src/zoda/babybear.rs) and cannot be compiled here, so each function below
 * restates one reference function and names it. Arithmetic is done exactly
 * the way the reference does it: canonical u32 values, products reduced with
 * `%` in 64 bits, a recursive even/odd reordering, radix-2 DIT stages, and
 * roots of unity derived from the smallest multiplicative generator.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ZO_P 2013265921u /* src/field/babybear.rs:9 */

/* ---- field (src/field/babybear.rs:19-78) ------------------------------- */

uint32_t zo_bb_new(uint64_t v) { return (uint32_t)(v % ZO_P); } /* :19-23 */
uint32_t zo_bb_add(uint32_t a, uint32_t b) {                     /* :45-52 */
    uint32_t s = a + b;
    return s >= ZO_P ? s - ZO_P : s;
}
uint32_t zo_bb_sub(uint32_t a, uint32_t b) { /* :58-66 */
    return a >= b ? a - b : a + ZO_P - b;
}
uint32_t zo_bb_mul(uint32_t a, uint32_t b) { /* :72-78 */
    return (uint32_t)(((uint64_t)a * b) % ZO_P);
}

/* ---- number theory (src/ntt/cpu.rs:62-110) ------------------------------ */

/* src/ntt/cpu.rs:62-71: square-and-multiply with `%` after every product. */
uint32_t zo_pow_mod(uint32_t b, uint32_t e, uint32_t p) {
    uint32_t r = 1u;
    b %= p;
    while (e > 0) {
        if (e & 1u) r = (uint32_t)(((uint64_t)r * b) % p);
        b = (uint32_t)(((uint64_t)b * b) % p);
        e >>= 1;
    }
    return r;
}

/* src/ntt/cpu.rs:73-86: distinct prime factors by trial division. */
static int zo_prime_factors(uint32_t m, uint32_t out[32]) {
    int cnt = 0;
    for (uint32_t q = 2; (uint64_t)q * q <= m; q++) {
        if (m % q == 0) {
            out[cnt++] = q;
            while (m % q == 0) m /= q;
        }
    }
    if (m > 1) out[cnt++] = m;
    return cnt;
}

/* src/ntt/cpu.rs:88-94: smallest g with g^((p-1)/q) != 1 for every prime q | p-1. */
uint32_t zo_find_generator(uint32_t p) {
    uint32_t f[32];
    int nf = zo_prime_factors(p - 1, f);
    for (uint32_t g = 2; g < p; g++) {
        int ok = 1;
        for (int i = 0; i < nf && ok; i++)
            if (zo_pow_mod(g, (p - 1) / f[i], p) == 1) ok = 0;
        if (ok) return g;
    }
    return 0; /* p not prime */
}

/* src/ntt/cpu.rs:96-110: roots[i] = omega^i, omega = g^((p-1)/n).
 * Returns 0 on success, -1 when n does not divide p-1 (the reference asserts). */
int zo_roots_of_unity(uint32_t n, uint32_t p, uint32_t* roots) {
    if (n < 1 || (p - 1) % n != 0) return -1;
    uint32_t g = zo_find_generator(p);
    uint32_t omega = zo_pow_mod(g, (p - 1) / n, p);
    uint32_t cur = 1;
    for (uint32_t i = 0; i < n; i++) {
        roots[i] = cur;
        cur = (uint32_t)(((uint64_t)cur * omega) % p);
    }
    return 0;
}

/* ---- transforms (src/ntt/cpu.rs:1-60) ------------------------------------ */

/* src/ntt/cpu.rs:34-46: reverse(values) = reverse(evens) ++ reverse(odds).
 * The reference builds new vectors per level; this walks the same recursion
 * with a stride instead, writing the reordered values into dst. */
static void zo_reverse_rec(const uint32_t* src, size_t stride, size_t n, uint32_t* dst) {
    if (n == 0) return;
    if (n == 1) {
        dst[0] = src[0];
        return;
    }
    size_t n_even = (n + 1) / 2; /* step_by(2) from index 0 */
    zo_reverse_rec(src, stride * 2, n_even, dst);
    zo_reverse_rec(src + stride, stride * 2, n / 2, dst + n_even);
}

/* src/ntt/cpu.rs:1-32: coeffs = reverse(values), then radix-2 stages with
 * len = 2, 4, ..., n; butterfly j of a block uses roots[j * (n / len)].
 * In place on values[0..n); scratch must hold n u32. */
static void zo_ntt_with_scratch(uint32_t* values, const uint32_t* roots, size_t n, uint32_t p,
                                uint32_t* scratch) {
    zo_reverse_rec(values, 1, n, scratch);
    memcpy(values, scratch, n * sizeof(uint32_t));
    for (size_t len = 2; len <= n; len *= 2) {
        size_t half = len / 2, stride = n / len;
        for (size_t blk = 0; blk + len <= n; blk += len) {
            uint32_t* lo = values + blk;
            uint32_t* hi = lo + half;
            for (size_t j = 0; j < half; j++) {
                uint64_t w = roots[j * stride];
                uint32_t a = lo[j];
                uint32_t b = (uint32_t)(((uint64_t)hi[j] * w) % p);
                lo[j] = (a + b) % p;
                hi[j] = (a + p - b) % p;
            }
        }
    }
}

int zo_ntt(uint32_t* values, const uint32_t* roots, size_t n, uint32_t p) {
    uint32_t* scratch = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    if (!scratch) return -1;
    zo_ntt_with_scratch(values, roots, n, p, scratch);
    free(scratch);
    return 0;
}

/* src/ntt/cpu.rs:48-60: ntt with inv_roots = [roots[0], roots[n-1], ..., roots[1]]
 * then every coefficient times n^(p-2). */
static void zo_intt_with_scratch(uint32_t* values, const uint32_t* roots, size_t n, uint32_t p,
                                 uint32_t* inv_roots, uint32_t* scratch) {
    inv_roots[0] = roots[0];
    for (size_t i = 1; i < n; i++) inv_roots[i] = roots[n - i];
    zo_ntt_with_scratch(values, inv_roots, n, p, scratch);
    uint64_t n_inv = zo_pow_mod((uint32_t)n, p - 2, p);
    for (size_t i = 0; i < n; i++) values[i] = (uint32_t)((values[i] * n_inv) % p);
}

int zo_intt(uint32_t* values, const uint32_t* roots, size_t n, uint32_t p) {
    uint32_t* buf = (uint32_t*)malloc(2 * (n ? n : 1) * sizeof(uint32_t));
    if (!buf) return -1;
    zo_intt_with_scratch(values, roots, n, p, buf, buf + n);
    free(buf);
    return 0;
}

static int zo_is_pow2(size_t n) { return n && !(n & (n - 1)); }

/* src/ntt/cpu.rs:132-152: BabyBear adapters; the roots are rebuilt per call. */
int zo_ntt_babybear(uint32_t* values, size_t n) {
    if (!zo_is_pow2(n)) return -1;
    uint32_t* roots = (uint32_t*)malloc(n * sizeof(uint32_t));
    if (!roots) return -1;
    zo_roots_of_unity((uint32_t)n, ZO_P, roots);
    int rc = zo_ntt(values, roots, n, ZO_P);
    free(roots);
    return rc;
}
int zo_intt_babybear(uint32_t* values, size_t n) {
    if (!zo_is_pow2(n)) return -1;
    uint32_t* roots = (uint32_t*)malloc(n * sizeof(uint32_t));
    if (!roots) return -1;
    zo_roots_of_unity((uint32_t)n, ZO_P, roots);
    int rc = zo_intt(values, roots, n, ZO_P);
    free(roots);
    return rc;
}

/* ---- ZODA extension (src/zoda/babybear.rs:34-46, CPU branch) ------------- */

static size_t zo_next_pow2(size_t x) {
    size_t r = 1;
    while (r < x) r <<= 1;
    return r;
}

/* One column, column-major: poly[0..n_kn) with the data in poly[0..n_k).
 * intt over the first n_k values, then ntt over all n_kn values
 * (src/zoda/babybear.rs:41-44). Tables come in precomputed so that the
 * column-parallel driver does not rebuild them per column. */
static void zo_extend_one(uint32_t* poly, size_t n_k, size_t n_kn, const uint32_t* roots_k,
                          const uint32_t* roots_kn, uint32_t* tmp /* 2*n_kn */) {
    zo_intt_with_scratch(poly, roots_k, n_k, ZO_P, tmp, tmp + n_kn);
    zo_ntt_with_scratch(poly, roots_kn, n_kn, ZO_P, tmp);
}

/* src/zoda/babybear.rs:40-45: every n_kn-long column of a column-major buffer.
 * threads <= 0 means "all OpenMP threads". Returns 0 or -1. */
int zo_extend_colmajor(uint32_t* square, size_t n_k, size_t n_kn, size_t cols, int threads) {
    if (!zo_is_pow2(n_k) || !zo_is_pow2(n_kn) || n_kn < n_k) return -1;
    uint32_t* roots_k = (uint32_t*)malloc(n_k * sizeof(uint32_t));
    uint32_t* roots_kn = (uint32_t*)malloc(n_kn * sizeof(uint32_t));
    if (!roots_k || !roots_kn) return -1;
    zo_roots_of_unity((uint32_t)n_k, ZO_P, roots_k);
    zo_roots_of_unity((uint32_t)n_kn, ZO_P, roots_kn);
    int err = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(| : err)
#endif
    {
        uint32_t* tmp = (uint32_t*)malloc(2 * n_kn * sizeof(uint32_t));
        if (!tmp) err = 1;
        else {
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (long long c = 0; c < (long long)cols; c++)
                zo_extend_one(square + (size_t)c * n_kn, n_k, n_kn, roots_k, roots_kn, tmp);
            free(tmp);
        }
    }
    free(roots_k);
    free(roots_kn);
    return err ? -1 : 0;
}

/* The encode of src/benchmarks/utils.rs:100-146 with CPU transforms:
 * row-major input[k][cols] -> transpose into zero-padded n_kn-tall columns ->
 * intt(n_k) -> ntt(n_kn) -> written back row-major out[n_out][cols], where
 * n_k = next_pow2(k), n_kn = next_pow2(k + n) (utils.rs:42-48) and
 * n_out = k + n rows are kept (the rows utils.rs:167-168 gathers).
 * col0/ncols select a column window of the square (the CPU baseline times a
 * bounded sample of columns); out then has ncols columns per row. */
int zo_encode_rowmajor(const uint32_t* in, uint32_t* out, size_t k, size_t n, size_t cols,
                       size_t col0, size_t ncols, int threads) {
    size_t n_k = zo_next_pow2(k), n_kn = zo_next_pow2(k + n), n_out = k + n;
    if (k == 0 || col0 + ncols > cols) return -1;
    uint32_t* roots_k = (uint32_t*)malloc(n_k * sizeof(uint32_t));
    uint32_t* roots_kn = (uint32_t*)malloc(n_kn * sizeof(uint32_t));
    if (!roots_k || !roots_kn) return -1;
    zo_roots_of_unity((uint32_t)n_k, ZO_P, roots_k);
    zo_roots_of_unity((uint32_t)n_kn, ZO_P, roots_kn);
    int err = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(| : err)
#endif
    {
        uint32_t* col = (uint32_t*)malloc(3 * n_kn * sizeof(uint32_t));
        if (!col) err = 1;
        else {
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (long long c = 0; c < (long long)ncols; c++) {
                size_t gc = col0 + (size_t)c;
                for (size_t r = 0; r < k; r++) col[r] = in[r * cols + gc];
                for (size_t r = k; r < n_kn; r++) col[r] = 0;
                zo_extend_one(col, n_k, n_kn, roots_k, roots_kn, col + n_kn);
                for (size_t r = 0; r < n_out; r++) out[r * ncols + (size_t)c] = col[r];
            }
            free(col);
        }
    }
    free(roots_k);
    free(roots_kn);
    return err ? -1 : 0;
}

/* ---- legacy FFI semantics (cuda/ntt_kernel.cu:184-208, src/ntt/cuda.rs:99-131)
 * cuda_ntt/cuda_intt transform, in place, the first n values of each of
 * `polys` polynomials laid stride apart; values past n are untouched. These
 * CPU versions define what the GPU drop-in must return. */
int zo_ntt_polys(uint32_t* values, const uint32_t* roots, uint32_t n, uint32_t polys, uint32_t stride,
                 int inverse) {
    if (n == 0 || stride < n) return -1;
    uint32_t* buf = (uint32_t*)malloc(2 * (size_t)n * sizeof(uint32_t));
    if (!buf) return -1;
    for (uint32_t c = 0; c < polys; c++) {
        uint32_t* poly = values + (size_t)c * stride;
        if (inverse) zo_intt_with_scratch(poly, roots, n, ZO_P, buf, buf + n);
        else zo_ntt_with_scratch(poly, roots, n, ZO_P, buf);
    }
    free(buf);
    return 0;
}

int zo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
