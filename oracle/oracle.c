/*
 * CPU ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of lambda_vm's CPU proving path for the Goldilocks
 * STARK backend (field, FFT/LDE, Keccak commitments, Fiat-Shamir transcript,
 * FRI, grinding, batch inversion, barycentric OOD, DEEP). It exists to check
 * the CUDA kernels in lambda_vm_b200/csrc; nothing in the product path links,
 * loads or calls it. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may use it.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths relative to the lambda_vm project root). The reference is Rust and
 * cannot be compiled in this environment, so parity of this oracle with the
 * reference is pinned by the reference's own known-answer tests (Keccak-256
 * vectors, the transcript KAT, closed-form NTT vectors, query-count formula);
 * see tests/golden/reference_kats.json and tests/test_oracle_kats.py.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

#define GL_P 0xFFFFFFFF00000001ULL
#define GL_EPS 0xFFFFFFFFULL

/* ------------------------------------------------------------------ */
/* Goldilocks field: crypto/math/src/field/goldilocks.rs:72-197        */
/* Values are u64 in [0, 2^64); results are reduced mod p but may be   */
/* non-canonical exactly like the reference (canonical only at I/O).   */
/* ------------------------------------------------------------------ */

uint64_t or_gl_canonical(uint64_t a) { return a >= GL_P ? a - GL_P : a; }

/* goldilocks.rs:80-96 */
uint64_t or_gl_add(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    int over = s < a;
    uint64_t s2 = s + (over ? GL_EPS : 0);
    int over2 = s2 < s;
    if (over2) s2 += GL_EPS;
    return s2;
}

/* goldilocks.rs:99-115 */
uint64_t or_gl_sub(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    int under = a < b;
    uint64_t d2 = d - (under ? GL_EPS : 0);
    int under2 = under && (d < GL_EPS);
    if (under2) d2 -= GL_EPS;
    return d2;
}

/* goldilocks.rs:196-216 (reduce128) */
static inline uint64_t reduce128(u128 x) {
    uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    uint64_t hh = hi >> 32, hl = hi & GL_EPS;
    uint64_t t0 = lo - hh;
    if (lo < hh) t0 -= GL_EPS;
    uint64_t t1 = (hl << 32) - hl;
    uint64_t r = t0 + t1;
    if (r < t0) r += GL_EPS;
    return r;
}

uint64_t or_gl_mul(uint64_t a, uint64_t b) { return reduce128((u128)a * b); }

/* goldilocks.rs:135-143 */
uint64_t or_gl_neg(uint64_t a) {
    uint64_t c = or_gl_canonical(a);
    return c == 0 ? 0 : GL_P - c;
}

uint64_t or_gl_pow(uint64_t a, uint64_t e) {
    uint64_t r = 1, b = a;
    while (e) {
        if (e & 1) r = or_gl_mul(r, b);
        b = or_gl_mul(b, b);
        e >>= 1;
    }
    return r;
}

/* goldilocks.rs:146-152: Fermat a^(p-2); returns 0 for a == 0 (caller checks) */
uint64_t or_gl_inv(uint64_t a) { return or_gl_pow(or_gl_canonical(a), GL_P - 2); }

/* crypto/math/src/field/traits.rs:83-95 with the generator at goldilocks.rs:540 */
uint64_t or_gl_root_of_unity(uint32_t log_n) {
    uint64_t r = 1753635133440165772ULL;
    if (log_n == 0) return 1;
    for (uint32_t i = 0; i < 32 - log_n; i++) r = or_gl_mul(r, r);
    return r;
}

/* ------------------------------------------------------------------ */
/* Fp3 = Fp[w]/(w^3 - 2): extensions_goldilocks.rs:280-420            */
/* ------------------------------------------------------------------ */
void or_fp3_mul(const uint64_t *a, const uint64_t *b, uint64_t *c) {
    /* c0 = a0b0 + 2(a1b2 + a2b1), c1 = a0b1 + a1b0 + 2a2b2, c2 = a0b2 + a1b1 + a2b0 */
    uint64_t b1_2 = or_gl_add(b[1], b[1]), b2_2 = or_gl_add(b[2], b[2]);
    uint64_t c0 = or_gl_add(or_gl_add(or_gl_mul(a[0], b[0]), or_gl_mul(a[1], b2_2)), or_gl_mul(a[2], b1_2));
    uint64_t c1 = or_gl_add(or_gl_add(or_gl_mul(a[0], b[1]), or_gl_mul(a[1], b[0])), or_gl_mul(a[2], b2_2));
    uint64_t c2 = or_gl_add(or_gl_add(or_gl_mul(a[0], b[2]), or_gl_mul(a[1], b[1])), or_gl_mul(a[2], b[0]));
    c[0] = c0; c[1] = c1; c[2] = c2;
}
void or_fp3_add(const uint64_t *a, const uint64_t *b, uint64_t *c) {
    for (int i = 0; i < 3; i++) c[i] = or_gl_add(a[i], b[i]);
}
void or_fp3_sub(const uint64_t *a, const uint64_t *b, uint64_t *c) {
    for (int i = 0; i < 3; i++) c[i] = or_gl_sub(a[i], b[i]);
}
/* extensions_goldilocks.rs:359-390 (norm-based inverse) */
int or_fp3_inv(const uint64_t *a, uint64_t *out) {
    uint64_t a0s = or_gl_mul(a[0], a[0]), a1s = or_gl_mul(a[1], a[1]), a2s = or_gl_mul(a[2], a[2]);
    uint64_t a0c = or_gl_mul(a0s, a[0]), a1c = or_gl_mul(a1s, a[1]), a2c = or_gl_mul(a2s, a[2]);
    uint64_t a012 = or_gl_mul(or_gl_mul(a[0], a[1]), a[2]);
    uint64_t a1c2 = or_gl_add(a1c, a1c);
    uint64_t a2c4 = or_gl_add(a2c, a2c); a2c4 = or_gl_add(a2c4, a2c4);
    uint64_t six = or_gl_add(or_gl_add(a012, a012), a012); six = or_gl_add(six, six);
    uint64_t norm = or_gl_sub(or_gl_add(or_gl_add(a0c, a1c2), a2c4), six);
    if (or_gl_canonical(norm) == 0) return -1;
    uint64_t ni = or_gl_inv(norm);
    uint64_t a1a2 = or_gl_mul(a[1], a[2]), a0a1 = or_gl_mul(a[0], a[1]), a0a2 = or_gl_mul(a[0], a[2]);
    out[0] = or_gl_mul(or_gl_sub(a0s, or_gl_add(a1a2, a1a2)), ni);
    out[1] = or_gl_mul(or_gl_sub(or_gl_add(a2s, a2s), a0a1), ni);
    out[2] = or_gl_mul(or_gl_sub(a1s, a0a2), ni);
    return 0;
}

/* ------------------------------------------------------------------ */
/* FFT: crypto/math/src/fft/two_half_fft.rs:51-236, bit_reversing.rs  */
/* ------------------------------------------------------------------ */
static inline uint64_t bitrev(uint64_t i, uint32_t log_n) {
    if (log_n == 0) return i;
    uint64_t r = 0;
    for (uint32_t b = 0; b < log_n; b++) r |= ((i >> b) & 1ULL) << (log_n - 1 - b);
    return r;
}

/* bit_reversing.rs: in_place_bit_reverse_permute_row_major */
static void bitrev_rows(uint64_t *buf, uint64_t n, uint64_t m, uint32_t log_n) {
    #pragma omp parallel for schedule(static) if (n * m > 65536)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint64_t j = bitrev((uint64_t)i, log_n);
        if (j > (uint64_t)i) {
            uint64_t *a = buf + (uint64_t)i * m, *b = buf + j * m;
            for (uint64_t c = 0; c < m; c++) { uint64_t t = a[c]; a[c] = b[c]; b[c] = t; }
        }
    }
}

static inline void dit_rows(uint64_t *lo, uint64_t *hi, uint64_t m, uint64_t tw) {
    for (uint64_t c = 0; c < m; c++) {
        uint64_t t = or_gl_mul(tw, hi[c]);
        uint64_t a = lo[c];
        lo[c] = or_gl_add(a, t);
        hi[c] = or_gl_sub(a, t);
    }
}

/* two_half_fft.rs:167-236: natural-order in, natural-order out, NOT scaled by
 * 1/n for the inverse direction (the LDE folds 1/n into its coset weights). */
int or_fft_two_half(uint64_t *buf, uint64_t n, uint64_t m, int inverse) {
    if (m == 0 || n == 0) return 0;
    if (n & (n - 1)) return -1;
    uint32_t log_n = 0;
    while ((1ULL << log_n) < n) log_n++;
    if (log_n == 0) return 0;
    if (log_n > 32) return -2;
    uint64_t half = n / 2;
    /* TwoHalfTwiddles::new (two_half_fft.rs:51-81) */
    uint64_t omega = or_gl_root_of_unity(log_n);
    if (inverse) omega = or_gl_inv(omega);
    uint64_t *tw = (uint64_t *)malloc(half * sizeof(uint64_t));
    uint64_t *btw = (uint64_t *)malloc(half * sizeof(uint64_t));
    uint64_t cur = 1;
    for (uint64_t i = 0; i < half; i++) { tw[i] = cur; cur = or_gl_mul(cur, omega); }
    uint32_t log_half = log_n - 1;
    for (uint64_t i = 0; i < half; i++) btw[i] = tw[bitrev(i, log_half)];
    uint32_t mid = (log_n + 1) / 2;

    bitrev_rows(buf, n, m, log_n);
    /* first half: layers 0..mid within 2^mid-row chunks (two_half_fft.rs:107-129) */
    uint64_t chunk_rows = 1ULL << mid;
    #pragma omp parallel for schedule(static) if (n * m > 65536)
    for (int64_t ch = 0; ch < (int64_t)(n / chunk_rows); ch++) {
        uint64_t *chunk = buf + (uint64_t)ch * chunk_rows * m;
        for (uint32_t layer = 0; layer < mid; layer++) {
            uint64_t hb = 1ULL << layer, block_rows = hb * 2, step = 1ULL << (log_n - 1 - layer);
            for (uint64_t b = 0; b < chunk_rows; b += block_rows)
                for (uint64_t j = 0; j < hb; j++)
                    dit_rows(chunk + (b + j) * m, chunk + (b + hb + j) * m, m, tw[j * step]);
        }
    }
    bitrev_rows(buf, n, m, log_n);
    /* second half: layers mid..log_n within 2^(log_n-mid)-row chunks (:133-155) */
    uint64_t chunk2 = 1ULL << (log_n - mid);
    #pragma omp parallel for schedule(static) if (n * m > 65536)
    for (int64_t th = 0; th < (int64_t)(n / chunk2); th++) {
        uint64_t *chunk = buf + (uint64_t)th * chunk2 * m;
        for (uint32_t layer = mid; layer < log_n; layer++) {
            uint64_t hb = 1ULL << (log_n - 1 - layer), block_rows = hb * 2;
            uint64_t first_block = (uint64_t)th << (layer - mid);
            for (uint64_t b = 0, bi = 0; b < chunk2; b += block_rows, bi++)
                for (uint64_t r = 0; r < hb; r++)
                    dit_rows(chunk + (b + r) * m, chunk + (b + hb + r) * m, m, btw[first_block + bi]);
        }
    }
    bitrev_rows(buf, n, m, log_n);
    free(tw); free(btw);
    return 0;
}

/* Coset weights g^i / n: crypto/stark/src/prover.rs:458-467 */
void or_coset_weights(uint64_t n, uint64_t offset, uint64_t *w) {
    uint64_t ninv = or_gl_inv(n % GL_P);
    uint64_t cur = ninv;
    for (uint64_t i = 0; i < n; i++) { w[i] = cur; cur = or_gl_mul(offset, cur); }
}

/* Polynomial::coset_lde_full_expand_row_major: crypto/math/src/polynomial.rs:527-608.
 * in: n*m row-major evaluations; out: (blowup*n)*m row-major, natural order. */
int or_coset_lde_row_major(const uint64_t *in, uint64_t n, uint64_t m, uint64_t blowup,
                           const uint64_t *weights, uint64_t *out) {
    if (m == 0 || n == 0) return 0;
    if ((n & (n - 1)) || (blowup & (blowup - 1)) || blowup == 0) return -1;
    uint64_t lde_n = n * blowup;
    memcpy(out, in, n * m * sizeof(uint64_t));
    int rc = or_fft_two_half(out, n, m, 1);
    if (rc) return rc;
    #pragma omp parallel for schedule(static) if (n * m > 65536)
    for (int64_t r = 0; r < (int64_t)n; r++)
        for (uint64_t c = 0; c < m; c++) out[r * m + c] = or_gl_mul(weights[r], out[r * m + c]);
    memset(out + n * m, 0, (lde_n - n) * m * sizeof(uint64_t));
    return or_fft_two_half(out, lde_n, m, 0);
}

/* ------------------------------------------------------------------ */
/* Keccak-f[1600] and Keccak-256 (0x01 padding). The permutation is    */
/* restated from the Keccak specification (FIPS 202 step mappings);    */
/* the reference uses sha3 0.10.8 / keccak 0.1.5 on the host            */
/* (crypto/crypto/src/hash/platform_keccak.rs) and an in-tree copy at   */
/* executor/src/vm/instruction/execution.rs:1001-1040.                 */
/* ------------------------------------------------------------------ */
static const uint64_t KRC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL, 0x8000000080008000ULL,
    0x000000000000808bULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008aULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800aULL, 0x800000008000000aULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

static inline uint64_t rotl(uint64_t x, unsigned r) { return r ? (x << r) | (x >> (64 - r)) : x; }

void or_keccak_f1600(uint64_t *A) {
    /* rho offsets r[x][y] computed from the (x,y) -> (y, 2x+3y) walk */
    static int init = 0;
    static unsigned R[25];
    if (!init) {
        unsigned x = 1, y = 0;
        R[0] = 0;
        for (unsigned t = 0; t < 24; t++) {
            R[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
            unsigned nx = y, ny = (2 * x + 3 * y) % 5;
            x = nx; y = ny;
        }
        init = 1;
    }
    for (int round = 0; round < 24; round++) {
        uint64_t C[5], D[5], B[25];
        for (int x = 0; x < 5; x++) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
        for (int x = 0; x < 5; x++) D[x] = C[(x + 4) % 5] ^ rotl(C[(x + 1) % 5], 1);
        for (int i = 0; i < 25; i++) A[i] ^= D[i % 5];
        /* rho + pi: B[y, 2x+3y] = rot(A[x,y], r[x,y]) */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(A[x + 5 * y], R[x + 5 * y]);
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++)
                A[x + 5 * y] = B[x + 5 * y] ^ ((~B[(x + 1) % 5 + 5 * y]) & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= KRC[round];
    }
}

/* Streaming Keccak-256 sponge (rate 136 bytes, pad 0x01 ... 0x80). */
typedef struct {
    uint64_t st[25];
    uint8_t buf[136];
    uint32_t pos;
} or_keccak_t;

void or_keccak_init(or_keccak_t *k) { memset(k, 0, sizeof(*k)); }

static void absorb_block(uint64_t *st, const uint8_t *blk) {
    for (int i = 0; i < 17; i++) {
        uint64_t v = 0;
        for (int b = 0; b < 8; b++) v |= (uint64_t)blk[8 * i + b] << (8 * b);
        st[i] ^= v;
    }
    or_keccak_f1600(st);
}

void or_keccak_update(or_keccak_t *k, const uint8_t *data, size_t len) {
    while (len) {
        size_t take = 136 - k->pos;
        if (take > len) take = len;
        memcpy(k->buf + k->pos, data, take);
        k->pos += (uint32_t)take; data += take; len -= take;
        if (k->pos == 136) { absorb_block(k->st, k->buf); k->pos = 0; }
    }
}

void or_keccak_final(const or_keccak_t *k0, uint8_t out[32]) {
    or_keccak_t k = *k0;
    memset(k.buf + k.pos, 0, 136 - k.pos);
    k.buf[k.pos] ^= 0x01;
    k.buf[135] ^= 0x80;
    absorb_block(k.st, k.buf);
    for (int i = 0; i < 4; i++)
        for (int b = 0; b < 8; b++) out[8 * i + b] = (uint8_t)(k.st[i] >> (8 * b));
}

void or_keccak256(const uint8_t *data, size_t len, uint8_t out[32]) {
    or_keccak_t k;
    or_keccak_init(&k);
    or_keccak_update(&k, data, len);
    or_keccak_final(&k, out);
}

/* ------------------------------------------------------------------ */
/* Merkle leaves over row-major LDE rows:                              */
/* crypto/stark/src/commitment.rs:52-107 (keccak_leaves_bit_reversed_  */
/* grouped) — leaf i hashes rows br(R*i) .. br(R*i+R-1), each row's     */
/* columns [col_start, col_end) in order, each element canonical, BE    */
/* (reference) or LE (little_endian != 0, the per-row LE variant).      */
/* row_u64 is the row stride in u64 (ext3 rows: 3 u64 per element).    */
/* ------------------------------------------------------------------ */
int or_leaves_row_major(const uint64_t *data, uint64_t num_rows, uint64_t row_u64, uint64_t col_start,
                        uint64_t col_end, uint32_t rows_per_leaf, int little_endian, uint8_t *out) {
    if (num_rows == 0) return 0;
    if (num_rows & (num_rows - 1)) return -1;
    if (rows_per_leaf == 0 || num_rows % rows_per_leaf) return -1;
    uint32_t log_n = 0;
    while ((1ULL << log_n) < num_rows) log_n++;
    uint64_t num_leaves = num_rows / rows_per_leaf;
    uint64_t width = col_end - col_start;
    #pragma omp parallel
    {
        uint8_t *buf = (uint8_t *)malloc(rows_per_leaf * width * 8 + 8);
        #pragma omp for schedule(static)
        for (int64_t li = 0; li < (int64_t)num_leaves; li++) {
            size_t off = 0;
            for (uint32_t k = 0; k < rows_per_leaf; k++) {
                uint64_t br = bitrev((uint64_t)li * rows_per_leaf + k, log_n);
                const uint64_t *row = data + br * row_u64;
                for (uint64_t c = col_start; c < col_end; c++) {
                    uint64_t v = or_gl_canonical(row[c]);
                    for (int b = 0; b < 8; b++)
                        buf[off + b] = (uint8_t)(little_endian ? (v >> (8 * b)) : (v >> (8 * (7 - b))));
                    off += 8;
                }
            }
            or_keccak256(buf, off, out + (uint64_t)li * 32);
        }
        free(buf);
    }
    return 0;
}

/* MerkleTree::build_from_hashed_leaves + utils::build:
 * crypto/crypto/src/merkle_tree/merkle.rs:201-225, utils.rs:52-96.
 * Leaves are padded to a power of two by repeating the last one; nodes has
 * 2L-1 entries of 32 bytes, root at 0, leaves at [L-1, 2L-1). Returns L. */
uint64_t or_merkle_build(const uint8_t *leaves, uint64_t num_leaves, uint8_t *nodes) {
    if (num_leaves == 0) return 0;
    uint64_t L = 1;
    while (L < num_leaves) L <<= 1;
    for (uint64_t i = 0; i < L; i++) {
        uint64_t src = i < num_leaves ? i : num_leaves - 1;
        memcpy(nodes + (L - 1 + i) * 32, leaves + src * 32, 32);
    }
    uint64_t begin = L - 1, end = 2 * begin;
    while (begin != end) {
        uint64_t nb = begin / 2, len = begin - nb;
        #pragma omp parallel for schedule(static) if (len > 4096)
        for (int64_t t = 0; t < (int64_t)len; t++) {
            or_keccak256(nodes + (begin + 2 * (uint64_t)t) * 32, 64, nodes + (nb + (uint64_t)t) * 32);
        }
        end = begin - 1;
        begin = nb;
    }
    return L;
}

/* MerkleTree::build_merkle_path (merkle.rs:260-280): sibling at each level,
 * leaf first. Returns the depth written. */
uint32_t or_merkle_path(const uint8_t *nodes, uint64_t leaves_len, uint64_t pos, uint8_t *out) {
    uint64_t node = pos + leaves_len - 1;
    uint32_t d = 0;
    while (node != 0) {
        uint64_t sib = (node % 2 == 0) ? node - 1 : node + 1;
        memcpy(out + (uint64_t)d * 32, nodes + sib * 32, 32);
        node = (node % 2 == 0) ? (node - 1) / 2 : node / 2;
        d++;
    }
    return d;
}

/* ------------------------------------------------------------------ */
/* Fiat-Shamir transcript: crypto/crypto/src/fiat_shamir/               */
/* default_transcript.rs:31-146 (Keccak hash chain + duplex buffer).    */
/* ------------------------------------------------------------------ */
typedef struct {
    or_keccak_t h;
    uint8_t out_buf[32];
    uint32_t out_pos;
} or_transcript_t;

size_t or_transcript_size(void) { return sizeof(or_transcript_t); }

void or_transcript_append(or_transcript_t *t, const uint8_t *data, size_t len) {
    t->out_pos = 32;
    or_keccak_update(&t->h, data, len);
}

void or_transcript_init(or_transcript_t *t, const uint8_t *data, size_t len) {
    or_keccak_init(&t->h);
    memset(t->out_buf, 0, 32);
    t->out_pos = 32;
    or_transcript_append(t, data, len);
}

/* default_transcript.rs:75-81: finalize_reset, reverse, absorb */
void or_transcript_sample(or_transcript_t *t, uint8_t out[32]) {
    uint8_t h[32];
    or_keccak_final(&t->h, h);
    for (int i = 0; i < 32; i++) out[i] = h[31 - i];
    or_keccak_init(&t->h);
    or_keccak_update(&t->h, out, 32);
    t->out_pos = 32;
}

/* default_transcript.rs:86-95 */
static uint64_t next_u64(or_transcript_t *t) {
    if (t->out_pos + 8 > 32) {
        or_transcript_sample(t, t->out_buf);
        t->out_pos = 0;
    }
    uint64_t v = 0;
    for (int b = 0; b < 8; b++) v = (v << 8) | t->out_buf[t->out_pos + b];
    t->out_pos += 8;
    return v;
}

void or_transcript_state(const or_transcript_t *t, uint8_t out[32]) { or_keccak_final(&t->h, out); }

/* goldilocks.rs:548-555 rejection sampler */
uint64_t or_transcript_sample_base(or_transcript_t *t) {
    for (;;) {
        uint64_t c = next_u64(t);
        if (c < GL_P) return c;
    }
}
/* extensions_goldilocks.rs:575-581 */
void or_transcript_sample_ext3(or_transcript_t *t, uint64_t *out) {
    for (int i = 0; i < 3; i++) out[i] = or_transcript_sample_base(t);
}
/* default_transcript.rs:136-145 */
uint64_t or_transcript_sample_u64(or_transcript_t *t, uint64_t upper) {
    uint64_t thr = (0 - upper) % upper;
    for (;;) {
        uint64_t c = next_u64(t);
        if (c >= thr) return c % upper;
    }
}
/* Field elements are absorbed as canonical BE bytes (goldilocks.rs:470-478,
 * extensions_goldilocks.rs:548-560). */
void or_transcript_append_base(or_transcript_t *t, uint64_t v) {
    uint8_t b[8];
    v = or_gl_canonical(v);
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * (7 - i)));
    or_transcript_append(t, b, 8);
}
void or_transcript_append_ext3(or_transcript_t *t, const uint64_t *v) {
    uint8_t b[24];
    for (int k = 0; k < 3; k++) {
        uint64_t c = or_gl_canonical(v[k]);
        for (int i = 0; i < 8; i++) b[8 * k + i] = (uint8_t)(c >> (8 * (7 - i)));
    }
    or_transcript_append(t, b, 24);
}

/* ------------------------------------------------------------------ */
/* Grinding: crypto/stark/src/grinding.rs:6-104, smallest-nonce rule    */
/* (the sequential `find` at grinding.rs:54-56).                        */
/* ------------------------------------------------------------------ */
void or_grind_inner_hash(const uint8_t seed[32], uint8_t g, uint8_t out[32]) {
    static const uint8_t PREFIX[8] = {0x01, 0x23, 0x45, 0x67, 0x89, 0xab, 0xcd, 0xed};
    uint8_t d[41];
    memcpy(d, PREFIX, 8);
    memcpy(d + 8, seed, 32);
    d[40] = g;
    or_keccak256(d, 41, out);
}

int or_grind_is_valid(const uint8_t inner[32], uint64_t nonce, uint8_t g) {
    uint8_t d[40], h[32];
    memcpy(d, inner, 32);
    for (int i = 0; i < 8; i++) d[32 + i] = (uint8_t)(nonce >> (8 * (7 - i)));
    or_keccak256(d, 40, h);
    uint64_t head = 0;
    for (int i = 0; i < 8; i++) head = (head << 8) | h[i];
    uint64_t limit = (g >= 64) ? 1 : (1ULL << (64 - g));
    return head < limit;
}

uint64_t or_grind(const uint8_t seed[32], uint8_t g, uint64_t max_nonce) {
    uint8_t inner[32];
    or_grind_inner_hash(seed, g, inner);
    const uint64_t CH = 1u << 16;
    for (uint64_t base = 0; base < max_nonce; base += CH) {
        uint64_t best = UINT64_MAX;
        #pragma omp parallel for schedule(static) reduction(min : best)
        for (int64_t i = 0; i < (int64_t)CH; i++) {
            uint64_t nonce = base + (uint64_t)i;
            if (nonce < max_nonce && or_grind_is_valid(inner, nonce, g) && nonce < best) best = nonce;
        }
        if (best != UINT64_MAX) return best;
    }
    return UINT64_MAX;
}

/* ------------------------------------------------------------------ */
/* Batch inversion (Montgomery): FieldElement::inplace_batch_inverse    */
/* (crypto/math/src/field/element.rs) over Fp3, interleaved triples.    */
/* ------------------------------------------------------------------ */
int or_fp3_batch_inverse(uint64_t *a, uint64_t n) {
    if (n == 0) return 0;
    uint64_t *pre = (uint64_t *)malloc(3 * n * sizeof(uint64_t));
    pre[0] = a[0]; pre[1] = a[1]; pre[2] = a[2];
    for (uint64_t i = 1; i < n; i++) or_fp3_mul(pre + 3 * (i - 1), a + 3 * i, pre + 3 * i);
    uint64_t inv[3];
    if (or_fp3_inv(pre + 3 * (n - 1), inv)) { free(pre); return -1; }
    for (uint64_t i = n - 1; i > 0; i--) {
        uint64_t ai[3], t[3];
        or_fp3_mul(inv, pre + 3 * (i - 1), ai);
        or_fp3_mul(inv, a + 3 * i, t);
        memcpy(inv, t, 24);
        memcpy(a + 3 * i, ai, 24);
    }
    memcpy(a, inv, 24);
    free(pre);
    return 0;
}

/* ------------------------------------------------------------------ */
/* FRI fold: crypto/stark/src/fri/fri_functions.rs:15-61.               */
/* evals: 2h ext3 values in bit-reversed order (pairs (2j, 2j+1) are a   */
/* point and its negation); inv_tw[j] = 1/x_j for the first of each      */
/* pair. out[j] = (lo + hi) + zeta * inv_tw[j] * (lo - hi).             */
/* ------------------------------------------------------------------ */
void or_fri_fold(const uint64_t *evals, uint64_t h, const uint64_t *inv_tw, const uint64_t *zeta,
                 uint64_t *out) {
    #pragma omp parallel for schedule(static) if (h > 65536)
    for (int64_t j = 0; j < (int64_t)h; j++) {
        const uint64_t *lo = evals + 6 * j, *hi = evals + 6 * j + 3;
        uint64_t s[3], d[3], zd[3];
        or_fp3_add(lo, hi, s);
        or_fp3_sub(lo, hi, d);
        or_fp3_mul(zeta, d, zd);
        for (int k = 0; k < 3; k++) out[3 * j + k] = or_gl_add(s[k], or_gl_mul(inv_tw[j], zd[k]));
    }
}

/* ------------------------------------------------------------------ */
/* Denominators for barycentric (R3) and DEEP (R4):                    */
/* crypto/math-cuda/src/inverse.rs:226-300 (DenomSign), polynomial.rs   */
/* barycentric_inv_denoms (z - x), prover.rs R4 (x - z).               */
/* out[k*n + i] = sign ? x_i - z_k : z_k - x_i  (ext3, then inverted).  */
/* ------------------------------------------------------------------ */
int or_inv_denoms(const uint64_t *x, uint64_t n, const uint64_t *z, uint64_t K, int x_minus_z, uint64_t *out) {
    for (uint64_t k = 0; k < K; k++)
        for (uint64_t i = 0; i < n; i++) {
            uint64_t *o = out + 3 * (k * n + i);
            const uint64_t *zk = z + 3 * k;
            if (x_minus_z) {
                o[0] = or_gl_sub(x[i], zk[0]); o[1] = or_gl_neg(zk[1]); o[2] = or_gl_neg(zk[2]);
            } else {
                o[0] = or_gl_sub(zk[0], x[i]); o[1] = zk[1]; o[2] = zk[2];
            }
        }
    return or_fp3_batch_inverse(out, K * n);
}

/* Barycentric sums (interpolate_coset_eval_ext_with_g_n_inv's inner sum,  */
/* polynomial.rs:207-235; barycentric.cu:210-300):                        */
/*   out[(k*cols + c)] = sum_i points[i] * col_c(row i*row_stride) * invd[k][i] */
/* `data` is row-major (rows x row_u64); ext3 != 0 reads 3-u64 elements.   */
void or_barycentric_sums(const uint64_t *data, uint64_t row_u64, uint64_t row_stride, int ext3, uint64_t cols,
                         const uint64_t *points, const uint64_t *invd, uint64_t n, uint64_t K, uint64_t *out) {
    #pragma omp parallel for schedule(static) if (cols * n > 65536)
    for (int64_t c = 0; c < (int64_t)cols; c++) {
        for (uint64_t k = 0; k < K; k++) {
            uint64_t acc[3] = {0, 0, 0};
            for (uint64_t i = 0; i < n; i++) {
                const uint64_t *row = data + i * row_stride * row_u64;
                uint64_t pe[3];
                if (ext3) {
                    for (int q = 0; q < 3; q++) pe[q] = or_gl_mul(points[i], row[3 * c + q]);
                } else {
                    pe[0] = or_gl_mul(points[i], row[c]); pe[1] = 0; pe[2] = 0;
                }
                uint64_t t[3];
                or_fp3_mul(pe, invd + 3 * (k * n + i), t);
                or_fp3_add(acc, t, acc);
            }
            for (int q = 0; q < 3; q++) out[3 * (k * cols + c) + q] = acc[q];
        }
    }
}

/* DEEP composition per LDE row (deep.cu:30-115, prover.rs:2400-2608):      */
/*   r = sum_j g_j (H_j(x) - H_j(z^P)) inv_h[i]                               */
/*     + sum_{j,k} g'_{jk} (t_j(x) - t_j(z w^k)) inv_t[k][i]                  */
/* main: rows x m base; aux: rows x A ext3; parts: rows x P ext3 (row-major).  */
/* out is written in natural order.                                          */
void or_deep(const uint64_t *main, uint64_t m, const uint64_t *aux, uint64_t A, const uint64_t *parts, uint64_t P,
             uint64_t rows, const uint64_t *h_ood, const uint64_t *trace_ood, const uint64_t *gammas_h,
             const uint64_t *gammas_tr, const uint64_t *inv_h, const uint64_t *inv_t, uint64_t K, uint64_t *out) {
    #pragma omp parallel for schedule(static) if (rows > 4096)
    for (int64_t i = 0; i < (int64_t)rows; i++) {
        uint64_t res[3] = {0, 0, 0}, t[3], u[3];
        for (uint64_t j = 0; j < P; j++) {
            or_fp3_sub(parts + 3 * ((uint64_t)i * P + j), h_ood + 3 * j, t);
            or_fp3_mul(gammas_h + 3 * j, t, u);
            or_fp3_mul(u, inv_h + 3 * i, t);
            or_fp3_add(res, t, res);
        }
        for (uint64_t j = 0; j < m + A; j++) {
            uint64_t tv[3];
            if (j < m) { tv[0] = main[(uint64_t)i * m + j]; tv[1] = 0; tv[2] = 0; }
            else memcpy(tv, aux + 3 * ((uint64_t)i * A + (j - m)), 24);
            for (uint64_t k = 0; k < K; k++) {
                uint64_t idx = 3 * (j * K + k);
                or_fp3_sub(tv, trace_ood + idx, t);
                or_fp3_mul(gammas_tr + idx, t, u);
                or_fp3_mul(u, inv_t + 3 * (k * rows + (uint64_t)i), t);
                or_fp3_add(res, t, res);
            }
        }
        memcpy(out + 3 * i, res, 24);
    }
}

/* FRI layer leaves: Keccak256(e[2j] || e[2j+1]), each ext3 as 3 canonical BE
 * u64 (FieldElementPairBackend, field_element_vector.rs; keccak.cu:384). */
void or_fri_leaves(const uint64_t *evals, uint64_t h, uint8_t *out) {
    #pragma omp parallel for schedule(static) if (h > 4096)
    for (int64_t j = 0; j < (int64_t)h; j++) {
        uint8_t b[48];
        for (int q = 0; q < 6; q++) {
            uint64_t v = or_gl_canonical(evals[6 * j + q]);
            for (int x = 0; x < 8; x++) b[8 * q + x] = (uint8_t)(v >> (8 * (7 - x)));
        }
        or_keccak256(b, 48, out + 32 * (uint64_t)j);
    }
}

/* LogUp aux build: crypto/stark/src/lookup.rs:1660-1842 (term columns and the
 * accumulated column) with the CSR descriptor of math-cuda/src/logup.rs:26-44.
 * main: row-major n x m. aux out: row-major n x (n_committed + 1) ext3:
 * term columns [0, n_committed) then the accumulated column.
 * Returns the table contribution L in L_out. */
int or_logup_aux(const uint64_t *main, uint64_t n, uint64_t m, uint32_t K, const uint64_t *bus_ids,
                 const uint32_t *elem_off, const uint32_t *elem_alpha, const uint64_t *elem_const,
                 const uint32_t *term_off, const uint64_t *term_coef, const uint32_t *term_col, uint32_t n_out,
                 const uint32_t *out_off, const uint32_t *out_int, const uint64_t *mult_const,
                 const uint32_t *mterm_off, const uint64_t *mterm_coef, const uint32_t *mterm_col,
                 uint32_t n_committed, const uint64_t *alpha_pows, const uint64_t *z, uint64_t *aux, uint64_t *L_out) {
    uint64_t *fp = (uint64_t *)malloc(3 * (uint64_t)K * n * sizeof(uint64_t) + 8);
    uint64_t *rs = (uint64_t *)calloc(3 * n + 1, sizeof(uint64_t));
    uint64_t W = n_committed + 1;
    for (uint64_t r = 0; r < n; r++)
        for (uint32_t k = 0; k < K; k++) {
            uint64_t lc[3] = {bus_ids[k], 0, 0};
            for (uint32_t e = elem_off[k]; e < elem_off[k + 1]; e++) {
                uint64_t base = elem_const[e];
                for (uint32_t t = term_off[e]; t < term_off[e + 1]; t++)
                    base = or_gl_add(base, or_gl_mul(term_coef[t], main[r * m + term_col[t]]));
                const uint64_t *a = alpha_pows + 3 * elem_alpha[e];
                for (int q = 0; q < 3; q++) lc[q] = or_gl_add(lc[q], or_gl_mul(a[q], base));
            }
            uint64_t *f = fp + 3 * ((uint64_t)k * n + r);
            or_fp3_sub(z, lc, f);
        }
    if (K && or_fp3_batch_inverse(fp, (uint64_t)K * n)) { free(fp); free(rs); return -1; }
    for (uint64_t r = 0; r < n; r++)
        for (uint32_t c = 0; c < n_out; c++) {
            uint64_t term[3] = {0, 0, 0};
            for (uint32_t ki = out_off[c]; ki < out_off[c + 1]; ki++) {
                uint32_t k = out_int[ki];
                uint64_t mu = mult_const[k];
                for (uint32_t t = mterm_off[k]; t < mterm_off[k + 1]; t++)
                    mu = or_gl_add(mu, or_gl_mul(mterm_coef[t], main[r * m + mterm_col[t]]));
                const uint64_t *rc = fp + 3 * ((uint64_t)k * n + r);
                for (int q = 0; q < 3; q++) term[q] = or_gl_add(term[q], or_gl_mul(rc[q], mu));
            }
            if (c < n_committed) memcpy(aux + 3 * (r * W + c), term, 24);
            or_fp3_add(rs + 3 * r, term, rs + 3 * r);
        }
    uint64_t L[3] = {0, 0, 0};
    for (uint64_t r = 0; r < n; r++) or_fp3_add(L, rs + 3 * r, L);
    uint64_t ninv = or_gl_inv(n % GL_P), off[3];
    for (int q = 0; q < 3; q++) off[q] = or_gl_mul(L[q], ninv);
    uint64_t acc[3] = {0, 0, 0};
    for (uint64_t r = 0; r < n; r++) {
        memcpy(aux + 3 * (r * W + n_committed), acc, 24);
        or_fp3_add(acc, rs + 3 * r, acc);
        or_fp3_sub(acc, off, acc);
    }
    memcpy(L_out, L, 24);
    free(fp);
    free(rs);
    return 0;
}
