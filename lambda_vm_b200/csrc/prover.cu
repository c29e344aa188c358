// One table's rounds 2-4 as a single native call: the per-table body of the
// reference prover (crypto/stark/src/prover.rs:3603-3977 rounds 2-3,
// 4433-4620 round 4, fri/mod.rs:27-205 FRI commit and queries) driven from
// C++ over the library's own kernels, so that a table costs its GPU work plus
// a few microseconds of host work per Fiat-Shamir step, and concurrent table
// drivers run without any interpreter lock.
//
// Step order and transcript absorption are those of the host-side prover it
// replaces (aux root; beta; composition root; z; OOD values main+aux at z and
// z*w, parts at z^2; gamma; FRI roots with a zeta before each; terminal
// coefficients; grinding nonce; query indexes), so proofs are identical.
#include <string.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "fs.cuh"

namespace sg {
namespace {

constexpr uint64_t P = 0xFFFFFFFF00000001ULL;

struct E3 {
    uint64_t v[3];
};

E3 e3(uint64_t a, uint64_t b = 0, uint64_t c = 0) { return E3{{a, b, c}}; }
E3 e3_mul(const E3& a, const E3& b) {
    E3 r;
    sg_host_fp3_mul(a.v, b.v, r.v);
    return r;
}
E3 e3_sub(const E3& a, const E3& b) {
    E3 r;
    sg_host_fp3_sub(a.v, b.v, r.v);
    return r;
}
E3 e3_scale(const E3& a, uint64_t s) {
    return e3(sg_host_gl_mul(a.v[0], s), sg_host_gl_mul(a.v[1], s), sg_host_gl_mul(a.v[2], s));
}
E3 e3_pow(const E3& a, uint64_t e) {
    E3 r;
    sg_host_fp3_pow(a.v, e, r.v);
    return r;
}
E3 e3_canon(const E3& a) { return e3(sg_host_gl_canon(a.v[0]), sg_host_gl_canon(a.v[1]), sg_host_gl_canon(a.v[2])); }

uint64_t root_of_unity(uint32_t log_n) {
    uint64_t r = 1753635133440165772ULL;  // two-adic generator (traits.rs:83-95)
    for (uint32_t i = 0; i < 32 - log_n; ++i) r = sg_host_gl_mul(r, r);
    return log_n == 0 ? 1 : r;
}

uint64_t bitrev(uint64_t x, uint32_t bits) {
    uint64_t r = 0;
    for (uint32_t b = 0; b < bits; ++b) r |= ((x >> b) & 1ULL) << (bits - 1 - b);
    return r;
}

// (z^n - g^n) / (n g^n): the barycentric prefactor of
// interpolate_coset_eval_ext_with_g_n_inv (polynomial.rs:207-235).
E3 ood_scale(const E3& z, uint64_t n, uint64_t g) {
    const uint64_t gn = sg_host_gl_pow(g, n);
    const uint64_t s = sg_host_gl_mul(sg_host_gl_inv(n % P), sg_host_gl_inv(gn));
    return e3_scale(e3_sub(e3_pow(z, n), e3(gn)), s);
}

// Device buffers of one table's rounds, released on the table's stream on
// every exit path.
struct Bufs {
    Ctx* ctx;
    cudaStream_t st;
    std::vector<std::pair<void*, uint64_t>> held;
    void* alloc(uint64_t bytes, int* rc) {
        void* p = nullptr;
        if (*rc != SG_OK) return nullptr;
        *rc = dev_alloc(ctx, st, bytes ? bytes : 8, &p);
        if (*rc == SG_OK) held.push_back({p, bytes ? bytes : 8});
        return p;
    }
    void release(void* p) {
        for (size_t i = 0; i < held.size(); ++i) {
            if (held[i].first == p) {
                dev_free(ctx, st, p, held[i].second);
                held.erase(held.begin() + i);
                return;
            }
        }
    }
    ~Bufs() {
        for (auto& h : held) dev_free(ctx, st, h.first, h.second);
    }
};

// Leaves over row pairs (big-endian canonical bytes, the prover's commitment
// layout), tree and root.
int commit_rows(Ctx* ctx, cudaStream_t st, Bufs& b, const uint64_t* d_rows, uint64_t rows, uint64_t row_u64,
                uint8_t** nodes_out, uint8_t root[32]) {
    int rc = SG_OK;
    const uint64_t L = rows / 2;
    uint8_t* nodes = (uint8_t*)b.alloc((2 * L - 1) * 32, &rc);
    if (rc) return rc;
    SG_TRY(leaves_row_major(ctx, st, d_rows, rows, row_u64, 0, row_u64, 2, 0, nodes + (L - 1) * 32));
    SG_TRY(merkle_inner(ctx, st, nodes, L));
    SG_CUDA(cudaMemcpyAsync(root, nodes, 32, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    *nodes_out = nodes;
    return SG_OK;
}

void absorb_e3(sg_transcript* t, const E3& v) { sg_transcript_append_ext3(t, v.v); }

E3 sample_e3(sg_transcript* t) {
    E3 r;
    sg_transcript_sample_ext3(t, r.v);
    return r;
}

// c_i = o^-i / keep * sum_j v_j w^-ij over the keep-point sub-coset of the
// final codeword (coeffs_from_terminal_codeword, fri/terminal.rs:72-103).
void terminal_coeffs(const std::vector<uint64_t>& cw_br, uint64_t terminal_offset, uint32_t eff_k, uint64_t* out) {
    const uint64_t len = cw_br.size() / 3;
    const uint64_t keep = 1ULL << eff_k;
    const uint64_t blow = len / keep;
    const uint32_t lbits = (uint32_t)log2_exact(len);
    std::vector<E3> sub(keep);
    for (uint64_t mm = 0; mm < keep; ++mm) {
        const uint64_t r = bitrev(mm * blow, lbits);
        sub[mm] = e3(cw_br[3 * r] % P, cw_br[3 * r + 1] % P, cw_br[3 * r + 2] % P);
    }
    const uint64_t winv = keep > 1 ? sg_host_gl_inv(root_of_unity(eff_k)) : 1;
    const uint64_t oinv = sg_host_gl_inv(terminal_offset);
    uint64_t s = sg_host_gl_inv(keep % P);
    uint64_t wi = 1;  // w^-i
    for (uint64_t i = 0; i < keep; ++i) {
        E3 acc = e3(0);
        uint64_t wij = 1;  // w^-ij
        for (uint64_t j = 0; j < keep; ++j) {
            for (int c = 0; c < 3; ++c) acc.v[c] = sg_host_gl_add(acc.v[c], sg_host_gl_mul(sub[j].v[c], wij));
            wij = sg_host_gl_mul(wij, wi);
        }
        const E3 r = e3_canon(e3_scale(acc, s));
        memcpy(out + 3 * i, r.v, 24);
        s = sg_host_gl_mul(s, oinv);
        wi = sg_host_gl_mul(wi, winv);
    }
}

}  // namespace
}  // namespace sg

using namespace sg;

extern "C" int sg_table_proof_shape(const sg_table_job* j, sg_proof_shape* s) {
    SG_CHECK_ARG(j && s && j->logup, "null argument");
    const int log_n = log2_exact(j->n), log_b = log2_exact(j->blowup);
    SG_CHECK_ARG(log_n >= 1 && log_b >= 1, "n and blowup must be powers of two >= 2");
    const uint32_t log_N = (uint32_t)(log_n + log_b);
    const uint32_t terminal_log = (uint32_t)log_b + j->final_log_degree < log_N ? (uint32_t)log_b + j->final_log_degree
                                                                                  : log_N;
    s->aux_cols = j->logup->num_out_cols;
    s->total_folds = log_N - terminal_log;
    s->fri_layers = s->total_folds > 0 ? s->total_folds - 1 : 0;
    s->terminal_coeffs = 1u << (terminal_log - (uint32_t)log_b);
    s->depth = log_N - 1;
    uint64_t paths = 0;
    for (uint32_t l = 0; l < s->fri_layers; ++l) paths += (uint64_t)j->queries * (s->depth - 1 - l) * 32;
    s->fri_path_bytes = paths;
    return SG_OK;
}

extern "C" int sg_prove_table(sg_ctx* c, void* stream, sg_transcript* t, const sg_table_job* j, sg_table_proof* o) {
    SG_CHECK_ARG(c && t && j && o && j->logup && j->program, "null argument");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    cudaStream_t st = (cudaStream_t)stream;
    sg_proof_shape shp;
    SG_TRY(sg_table_proof_shape(j, &shp));
    const uint64_t n = j->n, m = j->m, B = j->blowup, N = n * B, g = j->coset_offset;
    const uint32_t log_n = (uint32_t)log2_exact(n), log_N = (uint32_t)log2_exact(N);
    const uint64_t A = shp.aux_cols, Q = j->queries;
    SG_CHECK_ARG(j->logup->num_committed + 1 == A, "LogUp output columns");
    Bufs bf{ctx, st, {}};
    int rc = SG_OK;
    // ---- aux (LogUp) + commit
    uint64_t* d_aux = (uint64_t*)bf.alloc(n * 3 * A * 8, &rc);
    if (rc) return rc;
    E3 Lc;
    SG_TRY(sg_logup_aux(c, st, j->d_trace, n, m, j->logup, j->alpha_pows, j->n_alpha, j->lookup_challenges, d_aux,
                        Lc.v));
    uint64_t* d_aux_lde = (uint64_t*)bf.alloc(N * 3 * A * 8, &rc);
    if (rc) return rc;
    SG_TRY(coset_lde(ctx, st, d_aux, n, 3 * A, B, j->d_weights, d_aux_lde));
    bf.release(d_aux);
    uint8_t* aux_nodes = nullptr;
    SG_TRY(commit_rows(ctx, st, bf, d_aux_lde, N, 3 * A, &aux_nodes, o->aux_root));
    sg_transcript_append(t, o->aux_root, 32);
    memcpy(o->table_contribution, e3_canon(Lc).v, 24);
    // ---- round 2: composition polynomial
    const E3 beta = sample_e3(t);
    const uint32_t nroots = j->program->num_roots;
    std::vector<uint64_t> coefs(3ull * (nroots + j->num_boundary));
    E3 pw = e3(1);
    for (uint32_t i = 0; i < nroots + j->num_boundary; ++i) {
        memcpy(&coefs[3 * i], pw.v, 24);
        pw = e3_mul(pw, beta);
    }
    const E3 offset = e3_scale(Lc, sg_host_gl_inv(n % P));
    sg_composition comp{};
    comp.beta_trans = coefs.data();
    comp.d_z_inv = j->d_z_inv;
    comp.z_len = B;
    comp.num_boundary = j->num_boundary;
    comp.b_col = j->b_col;
    comp.b_is_aux = j->b_is_aux;
    comp.b_value = j->b_value;
    comp.b_beta = coefs.data() + 3ull * nroots;
    comp.d_b_z_inv = j->d_b_z_inv;
    uint64_t* d_h = (uint64_t*)bf.alloc(N * 3 * 8, &rc);
    if (rc) return rc;
    SG_TRY(sg_eval_constraints(c, st, j->program, j->lookup_challenges, 2, j->alpha_pows, j->n_alpha, offset.v,
                               j->d_main_lde, m, d_aux_lde, A, N, B, &comp, d_h));
    uint64_t* d_halves = (uint64_t*)bf.alloc(N / 2 * 6 * 8, &rc);
    if (rc) return rc;
    SG_TRY(sg_decompose_d2(c, st, d_h, N, j->d_inv2x, d_halves));
    bf.release(d_h);
    uint64_t* d_parts = (uint64_t*)bf.alloc(N * 6 * 8, &rc);
    if (rc) return rc;
    SG_TRY(coset_lde(ctx, st, d_halves, N / 2, 6, 2, j->d_comp_weights, d_parts));
    bf.release(d_halves);
    uint8_t* comp_nodes = nullptr;
    SG_TRY(commit_rows(ctx, st, bf, d_parts, N, 6, &comp_nodes, o->comp_root));
    sg_transcript_append(t, o->comp_root, 32);
    // ---- round 3: out-of-domain evaluations by barycentric sums over rows i*B
    E3 z;
    sg_transcript_sample_z_ood(t, n, N, g, z.v);
    const E3 zw = e3_scale(z, root_of_unity(log_n));
    const E3 z2 = e3_mul(z, z);
    const E3 pts3[3] = {z, zw, z2};
    uint64_t zs[9];
    for (int k = 0; k < 3; ++k) memcpy(zs + 3 * k, pts3[k].v, 24);
    uint64_t* d_invd = (uint64_t*)bf.alloc(3 * n * 3 * 8, &rc);
    if (rc) return rc;
    int zero = 0;
    SG_TRY(sg_inv_denoms_ext3(c, st, j->d_pts_n, n, zs, 3, 0, d_invd, &zero));
    if (zero) {
        set_error("prove_table: z_ood lies in the trace coset");
        return SG_ERR_INVALID;
    }
    uint64_t* d_S = (uint64_t*)bf.alloc((2 * m + 2 * A + 2) * 3 * 8, &rc);
    if (rc) return rc;
    SG_TRY(sg_barycentric_sums(c, st, j->d_main_lde, m, B, 0, m, j->d_pts_n, d_invd, n, 2, d_S));
    SG_TRY(sg_barycentric_sums(c, st, d_aux_lde, 3 * A, B, 1, A, j->d_pts_n, d_invd, n, 2, d_S + 6 * m));
    SG_TRY(sg_barycentric_sums(c, st, d_parts, 6, B, 1, 2, j->d_pts_n, d_invd + 2 * n * 3, n, 1,
                               d_S + 6 * m + 6 * A));
    std::vector<uint64_t> S((2 * m + 2 * A + 2) * 3);
    SG_CUDA(cudaMemcpyAsync(S.data(), d_S, S.size() * 8, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    bf.release(d_invd);
    bf.release(d_S);
    // round 4's denominators depend on z only: they are inverted while the
    // host absorbs the OOD values and samples gamma below. A point lies in
    // the LDE coset g * <w_N> iff it is a base-field element c with
    // (c / g)^N = 1, checked here instead of by the inversion's flag (whose
    // read would wait for it).
    auto in_lde_coset = [&](const E3& p) {
        return p.v[1] % P == 0 && p.v[2] % P == 0 && sg_host_gl_pow(sg_host_gl_mul(p.v[0], sg_host_gl_inv(g)), N) == 1;
    };
    if (in_lde_coset(z2)) {
        set_error("prove_table: z^2 lies in the LDE coset");
        return SG_ERR_INVALID;
    }
    if (in_lde_coset(z) || in_lde_coset(zw)) {
        set_error("prove_table: z_ood lies in the LDE coset");
        return SG_ERR_INVALID;
    }
    uint64_t* d_inv_h = (uint64_t*)bf.alloc(N * 3 * 8, &rc);
    uint64_t* d_inv_t = (uint64_t*)bf.alloc(2 * N * 3 * 8, &rc);
    if (rc) return rc;
    SG_TRY(sg_inv_denoms_ext3(c, st, j->d_pts_N, N, z2.v, 1, 1, d_inv_h, nullptr));
    uint64_t zzw[6];
    memcpy(zzw, z.v, 24);
    memcpy(zzw + 3, zw.v, 24);
    SG_TRY(sg_inv_denoms_ext3(c, st, j->d_pts_N, N, zzw, 2, 1, d_inv_t, nullptr));
    const E3 sc[3] = {ood_scale(z, n, g), ood_scale(zw, n, g), ood_scale(z2, n, g)};
    const uint64_t W = m + A;
    for (int k = 0; k < 2; ++k) {
        for (uint64_t col = 0; col < W; ++col) {
            const uint64_t* sv = col < m ? &S[3 * (k * m + col)] : &S[6 * m + 3 * (k * A + (col - m))];
            const E3 v = e3_canon(e3_mul(sc[k], e3(sv[0], sv[1], sv[2])));
            memcpy(o->trace_ood + 3 * (k * W + col), v.v, 24);
            absorb_e3(t, v);
        }
    }
    for (int jp = 0; jp < 2; ++jp) {
        const uint64_t* sv = &S[6 * m + 6 * A + 3 * jp];
        const E3 v = e3_canon(e3_mul(sc[2], e3(sv[0], sv[1], sv[2])));
        memcpy(o->parts_ood + 3 * jp, v.v, 24);
        absorb_e3(t, v);
    }
    // ---- round 4: DEEP composition
    const E3 gamma = sample_e3(t);
    std::vector<uint64_t> gh(6), gt(3 * 2 * W), tood(3 * 2 * W);
    pw = e3(1);
    for (uint64_t i = 0; i < 2 + 2 * W; ++i) {
        if (i < 2)
            memcpy(&gh[3 * i], pw.v, 24);
        else
            memcpy(&gt[3 * (i - 2)], pw.v, 24);
        pw = e3_mul(pw, gamma);
    }
    for (uint64_t col = 0; col < W; ++col)
        for (int k = 0; k < 2; ++k) memcpy(&tood[3 * (2 * col + k)], o->trace_ood + 3 * (k * W + col), 24);
    uint64_t* d_deep = (uint64_t*)bf.alloc(N * 3 * 8, &rc);
    if (rc) return rc;
    SG_TRY(sg_deep_composition(c, st, j->d_main_lde, m, d_aux_lde, A, d_parts, 2, N, o->parts_ood, tood.data(),
                               gh.data(), gt.data(), 2, d_inv_h, d_inv_t, 1, d_deep));
    bf.release(d_inv_h);
    bf.release(d_inv_t);
    // ---- FRI commit phase. The transcript steps between layers (absorb a
    // root, sample the next challenge) run on the device on a copy of the
    // transcript, so every layer is enqueued without a host round trip; the
    // advanced transcript, the roots and the final codeword come back in one
    // copy (laid out state | roots | codeword in one device block).
    struct Layer {
        uint64_t* ev;
        uint64_t len;
        uint8_t* nodes;
        uint64_t leaves;
    };
    std::vector<Layer> layers;
    const uint64_t* ev = d_deep;
    uint64_t ev_len = N;
    const uint64_t* tw = j->d_tw0;
    uint64_t* own_tw = nullptr;
    const uint64_t state_bytes = (sizeof(fs::State) + 63) / 64 * 64, roots_bytes = 32ull * shp.fri_layers;
    const uint64_t final_len = shp.total_folds > 0 ? N >> shp.total_folds : 0;
    uint8_t* d_back = nullptr;
    uint64_t* d_zeta = nullptr;
    if (shp.total_folds > 0) {
        d_back = (uint8_t*)bf.alloc(state_bytes + roots_bytes + final_len * 24, &rc);
        d_zeta = (uint64_t*)bf.alloc(3 * 8, &rc);
        if (rc) return rc;
        SG_TRY(fri_state_load_dev(ctx, st, &t->s, d_back));
    }
    const uint8_t* prev_root = nullptr;
    for (uint32_t l = 0; l < shp.fri_layers; ++l) {
        const uint64_t h = ev_len / 2;
        uint64_t* ev2 = (uint64_t*)bf.alloc(h * 3 * 8, &rc);
        uint64_t* tw2 = (uint64_t*)bf.alloc((h / 2 ? h / 2 : 1) * 8, &rc);
        uint8_t* nodes = (uint8_t*)bf.alloc((2 * (h / 2) - 1) * 32, &rc);
        if (rc) return rc;
        const uint64_t nl = h / 2;
        SG_TRY(fri_challenge_dev(ctx, st, d_back, prev_root, l ? d_back + state_bytes + 32 * (l - 1) : nullptr,
                                 d_zeta));
        SG_TRY(fri_fold_dev(ctx, st, ev, h, tw, d_zeta, ev2, tw2, nodes + (nl - 1) * 32));
        SG_TRY(merkle_inner(ctx, st, nodes, nl));
        prev_root = nodes;
        if (own_tw) bf.release(own_tw);  // stream-ordered: the fold above has read it
        layers.push_back({ev2, h, nodes, nl});
        ev = ev2;
        ev_len = h;
        tw = own_tw = tw2;
    }
    std::vector<uint64_t> final_cw;
    if (shp.total_folds > 0) {
        const uint64_t h = ev_len / 2;
        uint64_t* evf = (uint64_t*)(d_back + state_bytes + roots_bytes);
        uint64_t* twf = (uint64_t*)bf.alloc((h / 2 ? h / 2 : 1) * 8, &rc);
        if (rc) return rc;
        SG_TRY(fri_challenge_dev(ctx, st, d_back, prev_root,
                                 prev_root ? d_back + state_bytes + roots_bytes - 32 : nullptr, d_zeta));
        SG_TRY(fri_fold_dev(ctx, st, ev, h, tw, d_zeta, evf, twf, nullptr));
        std::vector<uint8_t> back(state_bytes + roots_bytes + h * 24);
        SG_CUDA(cudaMemcpyAsync(back.data(), d_back, back.size(), cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        memcpy(&t->s, back.data(), sizeof(fs::State));
        memcpy(o->fri_roots, back.data() + state_bytes, roots_bytes);
        final_cw.resize(h * 3);
        memcpy(final_cw.data(), back.data() + state_bytes + roots_bytes, h * 24);
        bf.release(twf);
    } else {
        final_cw.resize(ev_len * 3);
        SG_CUDA(cudaMemcpyAsync(final_cw.data(), ev, ev_len * 24, cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
    }
    if (own_tw) bf.release(own_tw);
    const uint64_t term_off = sg_host_gl_pow(g, 1ULL << shp.total_folds);
    terminal_coeffs(final_cw, term_off, (uint32_t)log2_exact(shp.terminal_coeffs), o->fri_final);
    for (uint32_t i = 0; i < shp.terminal_coeffs; ++i) sg_transcript_append_ext3(t, o->fri_final + 3 * i);
    // ---- grinding (grinding.rs:45-104) and query indexes
    uint64_t nonce = 0;
    if (j->grinding) {
        uint8_t pre[8 + 32 + 1] = {0x01, 0x23, 0x45, 0x67, 0x89, 0xAB, 0xCD, 0xED};
        sg_transcript_state(t, pre + 8);
        pre[40] = (uint8_t)j->grinding;
        uint8_t inner[32];
        sg_keccak256(pre, sizeof(pre), inner);
        uint64_t lanes[4];
        memcpy(lanes, inner, 32);  // little-endian u64 lanes
        SG_TRY(sg_grind(c, st, lanes, (uint8_t)j->grinding, &nonce));
        uint8_t nb[8];
        for (int i = 0; i < 8; ++i) nb[i] = (uint8_t)(nonce >> (56 - 8 * i));
        sg_transcript_append(t, nb, 8);
    }
    *o->nonce = nonce;
    for (uint64_t q = 0; q < Q; ++q) o->iotas[q] = sg_transcript_sample_u64(t, N / 2);
    // ---- openings: one index upload, one kernel per request, copies straight to the caller's buffers
    const uint64_t F = layers.size();
    std::vector<uint32_t> idx(2 * Q + Q + F * (2 * Q + Q));
    uint64_t p = 0;
    const uint64_t rows_off = p;
    for (uint64_t q = 0; q < Q; ++q) {
        idx[p++] = (uint32_t)bitrev(2 * o->iotas[q], log_N);
        idx[p++] = (uint32_t)bitrev(2 * o->iotas[q] + 1, log_N);
    }
    const uint64_t leaf_off = p;
    for (uint64_t q = 0; q < Q; ++q) idx[p++] = (uint32_t)o->iotas[q];
    std::vector<uint64_t> lrow_off(F), lleaf_off(F);
    for (uint64_t l = 0; l < F; ++l) {
        lrow_off[l] = p;
        for (uint64_t q = 0; q < Q; ++q) {
            const uint64_t lf = o->iotas[q] >> (l + 1);
            idx[p++] = (uint32_t)(2 * lf);
            idx[p++] = (uint32_t)(2 * lf + 1);
        }
        lleaf_off[l] = p;
        for (uint64_t q = 0; q < Q; ++q) idx[p++] = (uint32_t)(o->iotas[q] >> (l + 1));
    }
    uint32_t* d_idx = (uint32_t*)bf.alloc(idx.size() * 4, &rc);
    const uint64_t D = shp.depth;
    const uint64_t ob_rows = 2 * Q * (m + 3 * A + 6) * 8, ob_paths = 3 * Q * D * 32;
    const uint64_t ob_fri = F * 2 * Q * 24 + shp.fri_path_bytes;
    uint8_t* d_open = (uint8_t*)bf.alloc(ob_rows + ob_paths + ob_fri, &rc);
    if (rc) return rc;
    SG_CUDA(cudaMemcpyAsync(d_idx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, st));
    uint8_t* w = d_open;
    struct Out {
        uint8_t* dev;
        void* host;
        uint64_t bytes;
    };
    std::vector<Out> outs;
    auto rows_req = [&](const uint64_t* mat, uint64_t cols, uint64_t nrows, uint64_t off, uint64_t cnt, void* host) {
        if (cnt == 0 || cols == 0) return SG_OK;
        SG_TRY(sg_gather_rows(c, st, mat, cols, nrows, 0, cols, d_idx + off, (uint32_t)cnt, (uint64_t*)w));
        outs.push_back({w, host, cnt * cols * 8});
        w += cnt * cols * 8;
        return SG_OK;
    };
    auto path_req = [&](const uint8_t* nodes, uint64_t leaves, uint64_t off, void* host) {
        const uint64_t depth = (uint64_t)log2_exact(leaves);
        if (Q == 0 || depth == 0) return SG_OK;
        SG_TRY(sg_merkle_gather_paths(c, st, nodes, leaves, d_idx + off, (uint32_t)Q, w));
        outs.push_back({w, host, Q * depth * 32});
        w += Q * depth * 32;
        return SG_OK;
    };
    SG_TRY(rows_req(j->d_main_lde, m, N, rows_off, 2 * Q, o->open_main));
    SG_TRY(rows_req(d_aux_lde, 3 * A, N, rows_off, 2 * Q, o->open_aux));
    SG_TRY(rows_req(d_parts, 6, N, rows_off, 2 * Q, o->open_parts));
    SG_TRY(path_req(j->d_main_nodes, j->main_leaves_len, leaf_off, o->path_main));
    SG_TRY(path_req(aux_nodes, N / 2, leaf_off, o->path_aux));
    SG_TRY(path_req(comp_nodes, N / 2, leaf_off, o->path_parts));
    uint8_t* fri_path_host = o->fri_paths;
    for (uint64_t l = 0; l < F; ++l) {
        SG_TRY(rows_req(layers[l].ev, 3, layers[l].len, lrow_off[l], 2 * Q, o->fri_open + l * 2 * Q * 3));
        SG_TRY(path_req(layers[l].nodes, layers[l].leaves, lleaf_off[l], fri_path_host));
        fri_path_host += Q * (uint64_t)log2_exact(layers[l].leaves) * 32;
    }
    for (auto& x : outs) SG_CUDA(cudaMemcpyAsync(x.host, x.dev, x.bytes, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return SG_OK;  // Bufs releases every device buffer on the stream
}
