/*
 * CPU oracle for the dense complex128 statevector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates the reference's CPU kernels so
 * that the CUDA product can be checked against them, and so that a CPU baseline
 * can be timed beside it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU legs load it; the product never links, imports or calls it.
 *
 * Each function cites the reference function it restates (paths are relative
 * to the dqsim project root).  Complex arithmetic follows num-complex 0.4:
 *   (a*b).re = a.re*b.re - a.im*b.im,  (a*b).im = a.re*b.im + a.im*b.re
 * and is compiled with -ffp-contract=off so no FMA changes the rounding.
 *
 * RNG: rand_chacha 0.3.1 ChaCha8Rng seeded by rand_core 0.6.4 seed_from_u64
 * (PCG32 expansion of the u64 into a 32-byte key), read through rand_core's
 * BlockRng::next_u64 and converted to f64 by rand 0.8's Standard
 * distribution ((u64 >> 11) * 2^-53).  These crates are not vendored in the
 * reference tree (Cargo.lock pins them); the block function is pinned by a
 * ChaCha20 comparison against the `cryptography` package in the tests, the
 * seed expansion and 8-round stream are restated from the published crates
 * and are not pinned by any reference output.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    double re, im;
} c128;

/* src/engine.rs:8-9 */
#define PAR_THRESHOLD 12
#define MAX_QUBITS 5
#define MAX_DIM (1 << MAX_QUBITS)

static inline c128 cmul(c128 a, c128 b) {
    c128 r;
    r.re = a.re * b.re - a.im * b.im;
    r.im = a.re * b.im + a.im * b.re;
    return r;
}
static inline c128 cadd(c128 a, c128 b) {
    c128 r;
    r.re = a.re + b.re;
    r.im = a.im + b.im;
    return r;
}
static inline double norm_sqr(c128 a) { return a.re * a.re + a.im * a.im; }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

/* control_masks, src/engine.rs:45-62 (validation is done by the caller). */
static void control_masks(const int* cq, const int* cv, int nc, uint64_t* mask, uint64_t* desired) {
    uint64_t m = 0, d = 0;
    for (int i = 0; i < nc; i++) {
        uint64_t bit = (uint64_t)1 << cq[i];
        m |= bit;
        if (cv[i]) d |= bit;
    }
    *mask = m;
    *desired = d;
}

/*
 * for_each_pair + apply_one_qubit_impl, src/engine.rs:65-128.
 * Every index i with bit `target` clear and (i & mask) == desired is paired
 * with i + 2^target and updated as (a, b) <- (u00 a + u01 b, u10 a + u11 b).
 * `is_x` selects apply_x (src/engine.rs:153-155): a swap of the pair.
 */
void orc_apply_one_qubit(c128* s, int n, int target, const c128* u, const int* cq, const int* cv,
                         int nc, int is_x, int parallel) {
    uint64_t mask, desired;
    control_masks(cq, cv, nc, &mask, &desired);
    const uint64_t half = (uint64_t)1 << target;
    const uint64_t pairs = ((uint64_t)1 << n) >> 1;
    const c128 u00 = u[0], u01 = u[1], u10 = u[2], u11 = u[3];
    parallel = parallel && n >= PAR_THRESHOLD;
#pragma omp parallel for schedule(static) if (parallel)
    for (int64_t jj = 0; jj < (int64_t)pairs; jj++) {
        uint64_t j = (uint64_t)jj;
        uint64_t i = ((j >> target) << (target + 1)) | (j & (half - 1));
        if ((i & mask) != desired) continue;
        c128 a = s[i], b = s[i + half];
        if (is_x) {
            s[i] = b;
            s[i + half] = a;
        } else {
            s[i] = cadd(cmul(u00, a), cmul(u01, b));
            s[i + half] = cadd(cmul(u10, a), cmul(u11, b));
        }
    }
}

/* apply_diagonal, src/engine.rs:158-181: amp[i] *= diag[j(i)], qubits[0] is the MSB of j. */
void orc_apply_diagonal(c128* s, int n, const int* qubits, int k, const c128* diag, int parallel) {
    const uint64_t len = (uint64_t)1 << n;
    parallel = parallel && n >= PAR_THRESHOLD;
#pragma omp parallel for schedule(static) if (parallel)
    for (int64_t ii = 0; ii < (int64_t)len; ii++) {
        uint64_t i = (uint64_t)ii;
        uint64_t j = 0;
        for (int t = 0; t < k; t++) j = (j << 1) | ((i >> qubits[t]) & 1);
        s[i] = cmul(s[i], diag[j]);
    }
}

/* apply_swap, src/engine.rs:184-241: exchange |..1_a..0_b..> and |..0_a..1_b..> under controls. */
void orc_apply_swap(c128* s, int n, int a, int b, const int* cq, const int* cv, int nc, int parallel) {
    uint64_t mask, desired;
    control_masks(cq, cv, nc, &mask, &desired);
    int lo = a < b ? a : b, hi = a < b ? b : a;
    const uint64_t low_bit = (uint64_t)1 << lo, high_bit = (uint64_t)1 << hi;
    const uint64_t quads = ((uint64_t)1 << n) >> 2;
    parallel = parallel && n >= PAR_THRESHOLD;
#pragma omp parallel for schedule(static) if (parallel)
    for (int64_t jj = 0; jj < (int64_t)quads; jj++) {
        uint64_t j = (uint64_t)jj;
        j = ((j >> lo) << (lo + 1)) | (j & (low_bit - 1));
        j = ((j >> hi) << (hi + 1)) | (j & (high_bit - 1));
        uint64_t x = j | low_bit;  /* low bit set, high bit clear */
        uint64_t y = j | high_bit; /* high bit set, low bit clear */
        if ((x & mask) != desired) continue;
        c128 t = s[x];
        s[x] = s[y];
        s[y] = t;
    }
}

/* insert_target_zeros, src/engine.rs:245-251 */
static inline uint64_t insert_target_zeros(uint64_t base, const int* sorted, int k) {
    for (int t = 0; t < k; t++) {
        uint64_t low = ((uint64_t)1 << sorted[t]) - 1;
        base = (base & low) | ((base & ~low) << 1);
    }
    return base;
}

/*
 * DenseLayout::new + DenseLayout::apply, src/engine.rs:266-347.
 * u is row-major dim x dim with qubits[0] the MSB of the matrix index.
 * Rows are accumulated from zero in column order, as the reference does.
 */
void orc_apply_dense(c128* s, int n, const int* qubits, int k, const c128* u, int parallel) {
    const int dim = 1 << k;
    uint64_t offsets[MAX_DIM];
    int sorted[MAX_QUBITS];
    for (int j = 0; j < dim; j++) {
        uint64_t off = 0;
        for (int bit = 0; bit < k; bit++) off |= (uint64_t)((j >> (k - 1 - bit)) & 1) << qubits[bit];
        offsets[j] = off;
    }
    for (int t = 0; t < k; t++) sorted[t] = qubits[t];
    for (int x = 1; x < k; x++)
        for (int y = x; y > 0 && sorted[y - 1] > sorted[y]; y--) {
            int tmp = sorted[y];
            sorted[y] = sorted[y - 1];
            sorted[y - 1] = tmp;
        }
    const uint64_t bases = ((uint64_t)1 << n) >> k;
    parallel = parallel && n >= PAR_THRESHOLD;
#pragma omp parallel for schedule(static) if (parallel)
    for (int64_t cc = 0; cc < (int64_t)bases; cc++) {
        c128 values[MAX_DIM], result[MAX_DIM];
        uint64_t base = insert_target_zeros((uint64_t)cc, sorted, k);
        for (int j = 0; j < dim; j++) values[j] = s[base | offsets[j]];
        for (int row = 0; row < dim; row++) {
            c128 acc = {0.0, 0.0};
            for (int col = 0; col < dim; col++) acc = cadd(acc, cmul(u[row * dim + col], values[col]));
            result[row] = acc;
        }
        for (int j = 0; j < dim; j++) s[base | offsets[j]] = result[j];
    }
}

/*
 * measure_qubit_impl, src/engine.rs:367-426, with the uniform draw supplied
 * by the caller.  Both branch probabilities are summed directly.  Returns the
 * outcome, or -1 for a nonfinite or zero norm (the reference panics there).
 * `reset` applies the X of a Reset (src/monolithic/statevector/execution.rs:334-344)
 * when the outcome is 1.
 */
int orc_measure(c128* s, int n, int qubit, double draw, int parallel, double* probs_out) {
    const uint64_t len = (uint64_t)1 << n;
    const uint64_t bit = (uint64_t)1 << qubit;
    double p0 = 0.0, p1 = 0.0;
    parallel = parallel && n >= PAR_THRESHOLD;
#pragma omp parallel for schedule(static) reduction(+ : p0, p1) if (parallel)
    for (int64_t ii = 0; ii < (int64_t)len; ii++) {
        double v = norm_sqr(s[ii]);
        if (((uint64_t)ii & bit) != 0)
            p1 += v;
        else
            p0 += v;
    }
    if (probs_out) {
        probs_out[0] = p0;
        probs_out[1] = p1;
    }
    double total = p0 + p1;
    if (!isfinite(total) || !(total > 0.0)) return -1;
    int outcome = draw < p1 / total ? 1 : 0;
    double scale = 1.0 / sqrt(outcome ? p1 : p0);
#pragma omp parallel for schedule(static) if (parallel)
    for (int64_t ii = 0; ii < (int64_t)len; ii++) {
        int b = (((uint64_t)ii & bit) != 0);
        if (b == outcome) {
            s[ii].re *= scale;
            s[ii].im *= scale;
        } else {
            s[ii].re = 0.0;
            s[ii].im = 0.0;
        }
    }
    return outcome;
}

/* marginal_probs, src/engine.rs:439-453; qubits[0] is the MSB of the output index. */
void orc_marginal_probs(const c128* s, int n, const int* qubits, int k, double* out) {
    const uint64_t len = (uint64_t)1 << n;
    int direct = (k == n);
    for (int t = 0; t < k && direct; t++)
        if (qubits[t] != n - 1 - t) direct = 0;
    if (direct) {
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
        for (int64_t i = 0; i < (int64_t)len; i++) out[i] = norm_sqr(s[i]);
        return;
    }
    memset(out, 0, sizeof(double) * ((size_t)1 << k));
    for (uint64_t i = 0; i < len; i++) {
        uint64_t j = 0;
        for (int t = 0; t < k; t++) j = (j << 1) | ((i >> qubits[t]) & 1);
        out[j] += norm_sqr(s[i]);
    }
}

/* |<a|b>|^2 as SimulationResult::fidelity, src/monolithic/statevector/simulator.rs:178-190 */
double orc_fidelity(const c128* a, const c128* b, uint64_t len) {
    c128 dot = {0.0, 0.0};
    for (uint64_t i = 0; i < len; i++) {
        c128 ca = {a[i].re, -a[i].im};
        dot = cadd(dot, cmul(ca, b[i]));
    }
    return norm_sqr(dot);
}

/* Serial CDF as run_shots builds it, src/monolithic/statevector/shots.rs:137-149.
 * Returns 0 on an invalid total. */
int orc_cdf_inplace(double* p, uint64_t len) {
    double total = 0.0;
    for (uint64_t i = 0; i < len; i++) {
        total += p[i];
        p[i] = total;
    }
    if (!isfinite(total) || total <= 0.0) return 0;
    for (uint64_t i = 0; i < len; i++) p[i] /= total;
    p[len - 1] = 1.0;
    return 1;
}

/* cdf.partition_point(|&p| p <= draw).min(len - 1), shots.rs:156 */
uint64_t orc_partition_point(const double* cdf, uint64_t len, double draw) {
    uint64_t lo = 0, hi = len;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] <= draw)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < len - 1 ? lo : len - 1;
}

/* ------------------------------------------------------------------------- */
/* ChaCha block function (RFC 8439 layout: words 12-13 a 64-bit block        */
/* counter, words 14-15 the stream id, as rand_chacha lays them out).        */
/* ------------------------------------------------------------------------- */
static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

#define QR(a, b, c, d)                                                                            \
    do {                                                                                          \
        a += b;                                                                                   \
        d ^= a;                                                                                   \
        d = rotl32(d, 16);                                                                        \
        c += d;                                                                                   \
        b ^= c;                                                                                   \
        b = rotl32(b, 12);                                                                        \
        a += b;                                                                                   \
        d ^= a;                                                                                   \
        d = rotl32(d, 8);                                                                         \
        c += d;                                                                                   \
        b ^= c;                                                                                   \
        b = rotl32(b, 7);                                                                         \
    } while (0)

void orc_chacha_block_words(const uint32_t in[16], int double_rounds, uint32_t out[16]) {
    uint32_t x[16];
    memcpy(x, in, sizeof(x));
    for (int r = 0; r < double_rounds; r++) {
        QR(x[0], x[4], x[8], x[12]);
        QR(x[1], x[5], x[9], x[13]);
        QR(x[2], x[6], x[10], x[14]);
        QR(x[3], x[7], x[11], x[15]);
        QR(x[0], x[5], x[10], x[15]);
        QR(x[1], x[6], x[11], x[12]);
        QR(x[2], x[7], x[8], x[13]);
        QR(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + in[i];
}

/* rand_core 0.6.4 SeedableRng::seed_from_u64: PCG32 output words fill the seed. */
void orc_seed_from_u64(uint64_t state, uint32_t key[8]) {
    const uint64_t MUL = 6364136223846793005ULL;
    const uint64_t INC = 11634580027462260723ULL;
    for (int i = 0; i < 8; i++) {
        state = state * MUL + INC;
        uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        key[i] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    }
}

/* Word w of the ChaCha8Rng stream keyed by seed_from_u64(seed) (stream 0). */
static uint32_t chacha8_word(const uint32_t key[8], uint64_t w) {
    uint32_t in[16], out[16];
    in[0] = 0x61707865u;
    in[1] = 0x3320646eu;
    in[2] = 0x79622d32u;
    in[3] = 0x6b206574u;
    for (int i = 0; i < 8; i++) in[4 + i] = key[i];
    uint64_t block = w >> 4;
    in[12] = (uint32_t)block;
    in[13] = (uint32_t)(block >> 32);
    in[14] = 0;
    in[15] = 0;
    orc_chacha_block_words(in, 4, out);
    return out[w & 15];
}

/* k-th next_u64() of ChaCha8Rng::seed_from_u64(seed): words 2k (low) and 2k+1 (high). */
uint64_t orc_chacha8_u64(uint64_t seed, uint64_t k) {
    uint32_t key[8];
    orc_seed_from_u64(seed, key);
    uint64_t lo = chacha8_word(key, 2 * k), hi = chacha8_word(key, 2 * k + 1);
    return (hi << 32) | lo;
}

/* rand 0.8 Standard f64 from one next_u64. */
double orc_u64_to_f64(uint64_t v) { return (double)(v >> 11) * (1.0 / 9007199254740992.0); }

double orc_chacha8_f64(uint64_t seed, uint64_t k) { return orc_u64_to_f64(orc_chacha8_u64(seed, k)); }

/* First draw of seed_from_u64(seed0 + shot) for shot in [0, count): the
 * per-shot terminal-sampling draw of shots.rs:153-155. */
void orc_first_draws(uint64_t seed0, uint64_t start, uint64_t count, double* out) {
#pragma omp parallel for schedule(static) if (count >= 4096)
    for (int64_t i = 0; i < (int64_t)count; i++) out[i] = orc_chacha8_f64(seed0 + start + (uint64_t)i, 0);
}

/* count consecutive draws of one stream (SimulationResult.counts, engine.rs:490-491). */
void orc_stream_draws(uint64_t seed, uint64_t start, uint64_t count, double* out) {
    uint32_t key[8];
    orc_seed_from_u64(seed, key);
    for (uint64_t i = 0; i < count; i++) {
        uint64_t k = start + i;
        uint64_t lo = chacha8_word(key, 2 * k), hi = chacha8_word(key, 2 * k + 1);
        out[i] = orc_u64_to_f64((hi << 32) | lo);
    }
}
