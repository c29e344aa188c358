// Constraint evaluation (round 2) and the composition split for sm_100a.
//
// Reference behaviour:
//  * program format: crypto/stark/src/constraint_ir/device.rs (DeviceNode
//    {op, a, b, res}, OP_* tags, operand kind << 29 | payload, RES_EXT_BIT),
//    so a DeviceProgram lowered by the reference runs here unchanged;
//  * per-row semantics: eval_device_program (device.rs) / constraint_interp.cu
//    eval_program_row, with frame rows r = (row + offset * next_step) mod rows;
//  * composition: evaluator.rs accumulation,
//      H(row) = z_inv[row % z_len] * sum_c beta_c C_c(row)
//             + sum_b z_b_inv[b][row] * beta_b * (trace_b(row) - value_b);
//  * degree-2 split: prover.rs:1557-1662 decompose, H0 = (h(x)+h(-x))/2,
//    H1 = (h(x)-h(-x)) / (2x).
//
// Design: one thread per LDE row walks the program; its value slots (the
// lowering's max-live-set, base and ext classes) live in SHARED memory,
// laid out slot-major so a warp's accesses to one slot are consecutive.
// The reference keeps these slots in global memory, where their traffic
// dominates the walk. Trace reads come from the row-major resident LDEs.
//
// Streaming programs (lambda_vm_b200/ir.py lower(stream=True), node_roots
// set): trace values are OPK_VAR operands read where they are used instead of
// OP_VAR nodes holding a slot each, and every instruction that completes a
// constraint folds it into the row's composition sum (or writes it, in the
// per-constraint mode) at once, so no constraint holds a slot to the end of
// the walk. The slot file then holds only intermediates: a 2605-column AIR
// with 3434 constraints needs 101 words a row instead of 5719, which fits
// shared memory.
#include <vector>

#include "common.cuh"
#include "gl.cuh"
#include "cpu_air.cuh"
#include "keccak_air.cuh"

namespace sg {

using gl::fe3;

#define OP_CONST_BASE 0u
#define OP_CONST_EXT 1u
#define OP_VAR 2u
#define OP_RAP_CHALLENGE 3u
#define OP_ALPHA_POW 4u
#define OP_TABLE_OFFSET 5u
#define OP_ADD 6u
#define OP_SUB 7u
#define OP_MUL 8u
#define OP_NEG 9u
#define OP_EMBED 10u
#define OPK_SHIFT 29u
#define OPK_PAYLOAD_MASK 0x1FFFFFFFu
#define OPK_BASE_SLOT 0u
#define OPK_EXT_SLOT 1u
#define OPK_BASE_CONST 2u
#define OPK_EXT_CONST 3u
#define OPK_RAP 4u
#define OPK_ALPHA 5u
#define OPK_OFFSET 6u
#define OPK_VAR 7u
#define VAR_AUX_BIT (1u << 28)
#define VAR_OFF_SHIFT 20u
#define VAR_COL_MASK 0xFFFFFu
#define RES_EXT_BIT 0x80000000u
#define RES_SLOT_MASK 0x7FFFFFFFu
#define NO_ROOT 0xFFFFFFFFu

struct Uni {
    const uint64_t* base_consts;
    const uint64_t* ext_consts;  // 3 per entry
    const uint64_t* rap;
    const uint64_t* alpha;
    fe3 offset;
};

struct SlotFile {
    uint64_t* vb;  // base slot s at vb[s * st]
    uint64_t* ve;  // ext slot s component k at ve[(3s + k) * st]
    uint64_t st;
    __device__ __forceinline__ uint64_t gb(uint32_t s) const { return vb[(uint64_t)s * st]; }
    __device__ __forceinline__ void pb(uint32_t s, uint64_t v) const { vb[(uint64_t)s * st] = v; }
    __device__ __forceinline__ fe3 ge(uint32_t s) const {
        const uint64_t* p = ve + (uint64_t)s * 3 * st;
        return fe3{p[0], p[st], p[2 * st]};
    }
    __device__ __forceinline__ void pe(uint32_t s, fe3 v) const {
        uint64_t* p = ve + (uint64_t)s * 3 * st;
        p[0] = v.c0;
        p[st] = v.c1;
        p[2 * st] = v.c2;
    }
};

struct Trace {
    const uint64_t* main;
    uint64_t m;
    const uint64_t* aux;  // rows x A ext3
    uint64_t A;
    uint64_t rows;
    uint64_t next_step;
    const uint64_t* cm;   // the main LDE column-major (m x rows), or null
};

// One main-trace cell of an OPK_VAR operand: column-major when the copy
// exists (a warp's 32 rows are then one coalesced segment), else row-major.
__device__ __forceinline__ uint64_t main_cell(const Trace& t, uint64_t r, uint32_t col) {
    return t.cm ? t.cm[(uint64_t)col * t.rows + r] : t.main[r * t.m + col];
}

__device__ __forceinline__ bool is_base_kind(uint32_t enc) {
    const uint32_t k = enc >> OPK_SHIFT;
    return k == OPK_BASE_SLOT || k == OPK_BASE_CONST || (k == OPK_VAR && !(enc & VAR_AUX_BIT));
}
// frame row of an OPK_VAR operand
__device__ __forceinline__ uint64_t var_row(uint32_t p, const Trace& t, uint64_t row) {
    uint64_t r = row + (uint64_t)((p >> VAR_OFF_SHIFT) & 0xFFu) * t.next_step;
    return r >= t.rows ? r - t.rows : r;
}
__device__ __forceinline__ uint64_t base_op(uint32_t enc, const SlotFile& f, const Uni& u, const Trace& t,
                                            uint64_t row) {
    const uint32_t p = enc & OPK_PAYLOAD_MASK;
    switch (enc >> OPK_SHIFT) {
        case OPK_BASE_SLOT: return f.gb(p);
        case OPK_VAR: return main_cell(t, var_row(p, t, row), p & VAR_COL_MASK);
        default: return __ldg(u.base_consts + p);
    }
}
__device__ __forceinline__ fe3 ext_op(uint32_t enc, const SlotFile& f, const Uni& u, const Trace& t, uint64_t row) {
    const uint32_t p = enc & OPK_PAYLOAD_MASK;
    switch (enc >> OPK_SHIFT) {
        case OPK_BASE_SLOT: return fe3{f.gb(p), 0, 0};
        case OPK_EXT_SLOT: return f.ge(p);
        case OPK_BASE_CONST: return fe3{__ldg(u.base_consts + p), 0, 0};
        case OPK_EXT_CONST: return fe3{__ldg(u.ext_consts + 3 * p), __ldg(u.ext_consts + 3 * p + 1), __ldg(u.ext_consts + 3 * p + 2)};
        case OPK_RAP: return fe3{__ldg(u.rap + 3 * p), __ldg(u.rap + 3 * p + 1), __ldg(u.rap + 3 * p + 2)};
        case OPK_ALPHA: return fe3{__ldg(u.alpha + 3 * p), __ldg(u.alpha + 3 * p + 1), __ldg(u.alpha + 3 * p + 2)};
        case OPK_VAR: {
            const uint64_t r = var_row(p, t, row);
            if (!(p & VAR_AUX_BIT)) return fe3{main_cell(t, r, p & VAR_COL_MASK), 0, 0};
            const uint64_t* q = t.aux + (r * t.A + (p & VAR_COL_MASK)) * 3;
            return fe3{q[0], q[1], q[2]};
        }
        default: return u.offset;
    }
}

// Where a streaming walk puts each completed constraint: mode 0 folds
// beta_c * C_c into *sum; mode 1 writes C_c to out[c * rows + row].
struct Sink {
    const uint32_t* node_roots;  // null: roots pinned, combined after the walk
    const uint64_t* beta;
    int mode;
    uint64_t* out;
};

// A main-trace operand (OPK_VAR, not aux) is fetched PF nodes ahead of its
// node into a register ring, so its load latency overlaps the nodes between;
// every other operand is read where it is used.
__device__ __forceinline__ bool is_main_var(uint32_t enc) {
    return (enc >> OPK_SHIFT) == OPK_VAR && !(enc & VAR_AUX_BIT);
}
// operand k (1: a, 2: b) of node nd, when it is a main-trace read: only the
// operands of arithmetic nodes are operands (and validated as such)
__device__ __forceinline__ uint64_t prefetch(const uint4& nd, int k, const Trace& t, uint64_t row) {
    const bool arith = nd.x >= OP_ADD && nd.x <= (k == 1 ? OP_EMBED : OP_MUL);
    const uint32_t enc = k == 1 ? nd.y : nd.z;
    if (!arith || !is_main_var(enc)) return 0;
    const uint32_t p = enc & OPK_PAYLOAD_MASK;
    return main_cell(t, var_row(p, t, row), p & VAR_COL_MASK);
}
__device__ __forceinline__ uint64_t bop(uint32_t enc, uint64_t pv, const SlotFile& f, const Uni& u, const Trace& t,
                                        uint64_t row) {
    return is_main_var(enc) ? pv : base_op(enc, f, u, t, row);
}
__device__ __forceinline__ fe3 eop(uint32_t enc, uint64_t pv, const SlotFile& f, const Uni& u, const Trace& t,
                                   uint64_t row) {
    return is_main_var(enc) ? fe3{pv, 0, 0} : ext_op(enc, f, u, t, row);
}

// Node i of the walk; va, vb: the prefetched main-trace operands.
__device__ __forceinline__ void exec_node(const uint4 nd, uint32_t i, uint64_t va, uint64_t vb, const Uni& u,
                                          const SlotFile& f, const Trace& t, uint64_t row, const Sink& sk, fe3* sum) {
    const uint32_t slot = nd.w & RES_SLOT_MASK;
    const bool rx = (nd.w & RES_EXT_BIT) != 0;
    switch (nd.x) {
        case OP_VAR: {
            const uint32_t off = (nd.z >> 8) & 0xFFu;
            uint64_t r = row + (uint64_t)off * t.next_step;
            if (r >= t.rows) r -= t.rows;
            const uint32_t col = nd.y & 0xFFFFu;
            if ((nd.z >> 16) & 1u)
                f.pb(slot, main_cell(t, r, col));
            else {
                const uint64_t* p = t.aux + (r * t.A + col) * 3;
                f.pe(slot, fe3{p[0], p[1], p[2]});
            }
            break;
        }
        case OP_ADD:
            if (!rx)
                f.pb(slot, gl::add(bop(nd.y, va, f, u, t, row), bop(nd.z, vb, f, u, t, row)));
            else if (is_base_kind(nd.y)) {
                const uint64_t x = bop(nd.y, va, f, u, t, row);
                const fe3 y = eop(nd.z, vb, f, u, t, row);
                f.pe(slot, fe3{gl::add(x, y.c0), y.c1, y.c2});
            } else if (is_base_kind(nd.z)) {
                const fe3 x = eop(nd.y, va, f, u, t, row);
                f.pe(slot, fe3{gl::add(x.c0, bop(nd.z, vb, f, u, t, row)), x.c1, x.c2});
            } else
                f.pe(slot, gl::add3(eop(nd.y, va, f, u, t, row), eop(nd.z, vb, f, u, t, row)));
            break;
        case OP_SUB:
            if (!rx)
                f.pb(slot, gl::sub(bop(nd.y, va, f, u, t, row), bop(nd.z, vb, f, u, t, row)));
            else if (is_base_kind(nd.y)) {
                const uint64_t x = bop(nd.y, va, f, u, t, row);
                const fe3 y = eop(nd.z, vb, f, u, t, row);
                f.pe(slot, fe3{gl::sub(x, y.c0), gl::sub(0, y.c1), gl::sub(0, y.c2)});
            } else if (is_base_kind(nd.z)) {
                const fe3 x = eop(nd.y, va, f, u, t, row);
                f.pe(slot, fe3{gl::sub(x.c0, bop(nd.z, vb, f, u, t, row)), x.c1, x.c2});
            } else
                f.pe(slot, gl::sub3(eop(nd.y, va, f, u, t, row), eop(nd.z, vb, f, u, t, row)));
            break;
        case OP_MUL:
            if (!rx)
                f.pb(slot, gl::mul(bop(nd.y, va, f, u, t, row), bop(nd.z, vb, f, u, t, row)));
            else if (is_base_kind(nd.y))
                f.pe(slot, gl::mulb3(eop(nd.z, vb, f, u, t, row), bop(nd.y, va, f, u, t, row)));
            else if (is_base_kind(nd.z))
                f.pe(slot, gl::mulb3(eop(nd.y, va, f, u, t, row), bop(nd.z, vb, f, u, t, row)));
            else
                f.pe(slot, gl::mul3(eop(nd.y, va, f, u, t, row), eop(nd.z, vb, f, u, t, row)));
            break;
        case OP_NEG:
            if (!rx)
                f.pb(slot, gl::neg(bop(nd.y, va, f, u, t, row)));
            else {
                const fe3 x = eop(nd.y, va, f, u, t, row);
                f.pe(slot, fe3{gl::neg(x.c0), gl::neg(x.c1), gl::neg(x.c2)});
            }
            break;
        case OP_EMBED: f.pe(slot, eop(nd.y, va, f, u, t, row)); break;
        case OP_CONST_BASE: f.pb(slot, __ldg(u.base_consts + nd.y)); break;
        case OP_CONST_EXT: f.pe(slot, ext_op((OPK_EXT_CONST << OPK_SHIFT) | nd.y, f, u, t, row)); break;
        case OP_RAP_CHALLENGE: f.pe(slot, ext_op((OPK_RAP << OPK_SHIFT) | nd.y, f, u, t, row)); break;
        case OP_ALPHA_POW: f.pe(slot, ext_op((OPK_ALPHA << OPK_SHIFT) | nd.y, f, u, t, row)); break;
        case OP_TABLE_OFFSET: f.pe(slot, u.offset); break;
        default: break;
    }
    if (sk.node_roots) {
        const uint32_t c = __ldg(sk.node_roots + i);
        if (c != NO_ROOT) {
            if (sk.mode == 1) {
                const fe3 v = gl::canon3(rx ? f.ge(slot) : fe3{f.gb(slot), 0, 0});
                uint64_t* o = sk.out + 3 * ((uint64_t)c * t.rows + row);
                o[0] = v.c0;
                o[1] = v.c1;
                o[2] = v.c2;
            } else {
                const fe3 b{__ldg(sk.beta + 3 * c), __ldg(sk.beta + 3 * c + 1), __ldg(sk.beta + 3 * c + 2)};
                *sum = gl::add3(*sum, rx ? gl::mul3(b, f.ge(slot)) : gl::mulb3(b, f.gb(slot)));
            }
        }
    }
}

constexpr int PF = 1;             // prefetch distance, in nodes (1, 2, 4, 8 measured: 1 is fastest)
constexpr uint64_t CM_MIN_COLS = 32;  // narrower main LDEs are walked row-major

__device__ __forceinline__ void walk(const uint4* nodes, uint32_t num_nodes, const Uni& u, const SlotFile& f,
                                     const Trace& t, uint64_t row, const Sink& sk, fe3* sum) {
    uint4 q[PF];
    uint64_t pa[PF], pb[PF];
#pragma unroll
    for (int j = 0; j < PF; ++j) {
        q[j] = (uint32_t)j < num_nodes ? __ldg(nodes + j) : make_uint4(0xFFFFFFFFu, 0, 0, 0);
        pa[j] = prefetch(q[j], 1, t, row);
        pb[j] = prefetch(q[j], 2, t, row);
    }
    for (uint32_t i = 0; i < num_nodes; i += PF) {
#pragma unroll
        for (int j = 0; j < PF; ++j) {
            if (i + j < num_nodes) exec_node(q[j], i + j, pa[j], pb[j], u, f, t, row, sk, sum);
            const uint32_t nx = i + j + PF;
            q[j] = nx < num_nodes ? __ldg(nodes + nx) : make_uint4(0xFFFFFFFFu, 0, 0, 0);
            pa[j] = prefetch(q[j], 1, t, row);
            pb[j] = prefetch(q[j], 2, t, row);
        }
    }
}

__device__ __forceinline__ fe3 root_val(uint32_t enc, const SlotFile& f) {
    const uint32_t s = enc & RES_SLOT_MASK;
    return (enc & RES_EXT_BIT) ? f.ge(s) : fe3{f.gb(s), 0, 0};
}

struct Comp {
    const uint64_t* beta;     // num_roots ext3
    const uint64_t* z_inv;    // z_len base
    uint64_t z_len;
    uint32_t nb;              // boundary constraints
    const uint64_t* b_col;    // nb
    const uint64_t* b_aux;    // nb (0/1)
    const uint64_t* b_value;  // nb ext3
    const uint64_t* b_beta;   // nb ext3
    const uint64_t* b_zinv;   // nb x rows
};

// mode 0: composition H(row); mode 1: per-constraint matrix evals[c*rows + row].
__global__ void k_constraints(const uint4* nodes, uint32_t num_nodes, const uint32_t* roots, uint32_t num_roots,
                              const uint32_t* node_roots, uint32_t nbs, uint32_t nes, Uni u, Trace t, Comp cp,
                              int mode, uint64_t* out, uint64_t* gscratch, const uint64_t* extra) {
    extern __shared__ uint64_t shs[];
    const uint64_t T = blockDim.x;
    SlotFile f;
    if (gscratch) {
        const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
        const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        f.vb = gscratch + g;
        f.ve = gscratch + (uint64_t)nbs * nthreads + g;
        f.st = nthreads;
    } else {
        f.vb = shs + threadIdx.x;
        f.ve = shs + (uint64_t)nbs * T + threadIdx.x;
        f.st = T;
    }
    for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < t.rows;
         row += (uint64_t)gridDim.x * blockDim.x) {
        fe3 sum = extra ? fe3{extra[3 * row], extra[3 * row + 1], extra[3 * row + 2]} : fe3{0, 0, 0};
        walk(nodes, num_nodes, u, f, t, row, Sink{node_roots, cp.beta, mode, out}, &sum);
        if (node_roots && mode == 1) continue;
        if (mode == 1) {
            for (uint32_t c = 0; c < num_roots; ++c) {
                const fe3 v = gl::canon3(root_val(roots[c], f));
                uint64_t* o = out + 3 * ((uint64_t)c * t.rows + row);
                o[0] = v.c0;
                o[1] = v.c1;
                o[2] = v.c2;
            }
            continue;
        }
        for (uint32_t c = 0; node_roots == nullptr && c < num_roots; ++c) {
            const uint32_t enc = roots[c];
            const fe3 b{__ldg(cp.beta + 3 * c), __ldg(cp.beta + 3 * c + 1), __ldg(cp.beta + 3 * c + 2)};
            if (enc & RES_EXT_BIT)
                sum = gl::add3(sum, gl::mul3(b, f.ge(enc & RES_SLOT_MASK)));
            else
                sum = gl::add3(sum, gl::mulb3(b, f.gb(enc & RES_SLOT_MASK)));
        }
        fe3 h = gl::mulb3(sum, __ldg(cp.z_inv + row % cp.z_len));
        for (uint32_t b = 0; b < cp.nb; ++b) {
            const uint64_t col = cp.b_col[b];
            fe3 cell;
            if (cp.b_aux[b]) {
                const uint64_t* p = t.aux + (row * t.A + col) * 3;
                cell = fe3{p[0], p[1], p[2]};
            } else {
                cell = fe3{t.main[row * t.m + col], 0, 0};
            }
            const fe3 val{cp.b_value[3 * b], cp.b_value[3 * b + 1], cp.b_value[3 * b + 2]};
            const fe3 bb{cp.b_beta[3 * b], cp.b_beta[3 * b + 1], cp.b_beta[3 * b + 2]};
            const fe3 zb = gl::mulb3(bb, cp.b_zinv[(uint64_t)b * t.rows + row]);
            h = gl::add3(h, gl::mul3(zb, gl::sub3(cell, val)));
        }
        h = gl::canon3(h);
        out[3 * row] = h.c0;
        out[3 * row + 1] = h.c1;
        out[3 * row + 2] = h.c2;
    }
}

// The main LDE column-major for the walk: 32 x 32 tiles through shared memory,
// rows x m in, m x rows out. Grid: x = row tiles, y = column tiles.
__global__ void k_to_columns(const uint64_t* __restrict__ in, uint64_t rows, uint64_t m, uint64_t* __restrict__ out) {
    __shared__ uint64_t tile[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.x * 32, c0 = (uint64_t)blockIdx.y * 32;
    for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
        const uint64_t r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < m) tile[k][threadIdx.x] = in[r * m + c];
    }
    __syncthreads();
    for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
        const uint64_t c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < m) out[c * rows + r] = tile[threadIdx.x][k];
    }
}

// H0[i] = (h[i] + h[i+n]) / 2, H1[i] = inv_2x[i] (h[i] - h[i+n]); out rows: [H0 | H1] ext3.
__global__ void k_decompose_d2(const uint64_t* h, const uint64_t* inv_2x, uint64_t two_inv, uint64_t n,
                               uint64_t* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const fe3 x{h[3 * i], h[3 * i + 1], h[3 * i + 2]};
    const fe3 y{h[3 * (i + n)], h[3 * (i + n) + 1], h[3 * (i + n) + 2]};
    const fe3 a = gl::canon3(gl::mulb3(gl::add3(x, y), two_inv));
    const fe3 b = gl::canon3(gl::mulb3(gl::sub3(x, y), inv_2x[i]));
    uint64_t* o = out + 6 * i;
    o[0] = a.c0;
    o[1] = a.c1;
    o[2] = a.c2;
    o[3] = b.c0;
    o[4] = b.c1;
    o[5] = b.c2;
}

// ---- a table's LogUp constraints from its descriptor (lookup.rs:2185-2290)
// Interaction k's fingerprint fp_k = z - (bus_k + sum_e alpha^{ea_e}
// (c_e + sum_t coef_t main[col_t])) and signed multiplicity m_k = mc_k +
// sum_t mk_t main[ml_t] (the descriptor carries the sign). Committed column p
// holds the pair (2p, 2p+1): aux_p fa fb - ma fb - mb fa; the accumulated
// column, with delta = aux'_acc - aux_acc - sum_p aux_p + table_offset, is
// delta f - m over one remaining interaction or delta f1 f2 - m1 f2 - m2 f1
// over two.
struct LogupDev {
    const uint64_t *bus, *ec, *tc, *mc, *mk;
    const uint32_t *eo, *ea, *to, *tl, *mo, *ml;
    uint32_t K, nc;
};

// coef * x, without the product for the common coefficients 1 and -1 (the
// descriptor is the same for every thread, so the branch is uniform)
__device__ __forceinline__ uint64_t logup_scale(uint64_t coef, uint64_t x) {
    return coef == 1 ? x : coef == 0xFFFFFFFF00000000ULL ? gl::neg(x) : gl::mul(coef, x);
}

__device__ __forceinline__ fe3 logup_fp(const LogupDev& d, const Trace& t, uint64_t row, uint32_t k, fe3 z,
                                        const uint64_t* alpha) {
    gl::wacc3 acc = gl::wzero3();
    for (uint32_t e = __ldg(d.eo + k), e1 = __ldg(d.eo + k + 1); e < e1; ++e) {
        uint64_t v = __ldg(d.ec + e);
        for (uint32_t q = __ldg(d.to + e), q1 = __ldg(d.to + e + 1); q < q1; ++q)
            v = gl::add(v, logup_scale(__ldg(d.tc + q), main_cell(t, row, __ldg(d.tl + q))));
        const uint32_t ai = __ldg(d.ea + e);
        gl::wmacb3(acc, fe3{__ldg(alpha + 3 * ai), __ldg(alpha + 3 * ai + 1), __ldg(alpha + 3 * ai + 2)}, v);
    }
    const fe3 s = gl::wreduce3(acc);
    return fe3{gl::sub(gl::sub(z.c0, __ldg(d.bus + k)), s.c0), gl::sub(z.c1, s.c1), gl::sub(z.c2, s.c2)};
}

__device__ __forceinline__ uint64_t logup_mult(const LogupDev& d, const Trace& t, uint64_t row, uint32_t k) {
    uint64_t m = __ldg(d.mc + k);
    for (uint32_t q = __ldg(d.mo + k), q1 = __ldg(d.mo + k + 1); q < q1; ++q)
        m = gl::add(m, logup_scale(__ldg(d.mk + q), main_cell(t, row, __ldg(d.ml + q))));
    return m;
}

// mode 0: out[row] (+)= sum_c beta[root0 + c] C_c (add: out already holds the
// row's other constraints); mode 1: out[(root0 + c) * rows + row] = C_c.
__global__ void __launch_bounds__(128) k_logup_constraints(Trace t, LogupDev d, fe3 z, const uint64_t* alpha,
                                                           fe3 off, const uint64_t* beta, uint32_t root0, int mode,
                                                           int add, uint64_t* out) {
    for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < t.rows;
         row += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t rn = row + t.next_step >= t.rows ? row + t.next_step - t.rows : row + t.next_step;
        const uint64_t* ar = t.aux + row * t.A * 3;
        const uint64_t* an = t.aux + (rn * t.A + d.nc) * 3;
        fe3 sum{0, 0, 0};
        auto emit = [&](uint32_t c, const fe3& v) {
            if (mode == 1) {
                const fe3 w = gl::canon3(v);
                uint64_t* o = out + 3 * ((uint64_t)(root0 + c) * t.rows + row);
                o[0] = w.c0, o[1] = w.c1, o[2] = w.c2;
            } else {
                const uint64_t* b = beta + 3 * (uint64_t)(root0 + c);
                sum = gl::add3(sum, gl::mul3(fe3{__ldg(b), __ldg(b + 1), __ldg(b + 2)}, v));
            }
        };
        fe3 delta = gl::sub3(fe3{an[0], an[1], an[2]}, fe3{ar[3 * d.nc], ar[3 * d.nc + 1], ar[3 * d.nc + 2]});
        for (uint32_t p = 0; p < d.nc; ++p) {
            const fe3 ap{ar[3 * p], ar[3 * p + 1], ar[3 * p + 2]};
            delta = gl::sub3(delta, ap);
            const fe3 fa = logup_fp(d, t, row, 2 * p, z, alpha), fb = logup_fp(d, t, row, 2 * p + 1, z, alpha);
            const uint64_t ma = logup_mult(d, t, row, 2 * p), mb = logup_mult(d, t, row, 2 * p + 1);
            emit(p, gl::sub3(gl::sub3(gl::mul3(gl::mul3(ap, fa), fb), gl::mulb3(fb, ma)), gl::mulb3(fa, mb)));
        }
        delta = gl::add3(delta, off);
        const uint32_t k0 = 2 * d.nc;
        if (d.K == k0 + 1) {
            const fe3 f = logup_fp(d, t, row, k0, z, alpha);
            emit(d.nc, gl::sub3(gl::mul3(delta, f), fe3{logup_mult(d, t, row, k0), 0, 0}));
        } else {
            const fe3 f1 = logup_fp(d, t, row, k0, z, alpha), f2 = logup_fp(d, t, row, k0 + 1, z, alpha);
            const uint64_t m1 = logup_mult(d, t, row, k0), m2 = logup_mult(d, t, row, k0 + 1);
            emit(d.nc, gl::sub3(gl::sub3(gl::mul3(gl::mul3(delta, f1), f2), gl::mulb3(f2, m1)), gl::mulb3(f1, m2)));
        }
        if (mode == 0) {
            if (add) sum = gl::add3(sum, fe3{out[3 * row], out[3 * row + 1], out[3 * row + 2]});
            out[3 * row] = sum.c0, out[3 * row + 1] = sum.c1, out[3 * row + 2] = sum.c2;
        }
    }
}

// A descriptor the LogUp kernel can evaluate: CSR arrays in range for a main
// trace of m columns and n_alpha alpha powers, in the standard column layout.
static int check_logup_desc(const sg_logup_desc* d, uint64_t m, uint32_t n_alpha) {
    const uint32_t K = d->num_interactions, nc = d->num_committed;
    SG_CHECK_ARG(K >= 1 && d->bus_ids && d->elem_offsets && d->term_offsets && d->mult_consts && d->mult_term_offsets,
                 "logup: empty descriptor");
    SG_CHECK_ARG(K == 2 * nc + 1 || K == 2 * nc + 2, "logup: one or two interactions beyond the committed pairs");
    SG_CHECK_ARG(d->num_out_cols == nc + 1 && d->out_col_offsets && d->out_col_interactions,
                 "logup: committed columns plus one accumulated column");
    for (uint32_t o = 0; o <= nc; ++o)
        SG_CHECK_ARG(d->out_col_offsets[o] == 2 * o, "logup: committed columns hold interaction pairs");
    SG_CHECK_ARG(d->out_col_offsets[nc + 1] == K, "logup: the accumulated column holds the rest");
    for (uint32_t i = 0; i < K; ++i) SG_CHECK_ARG(d->out_col_interactions[i] == i, "logup: interactions in order");
    for (uint32_t k = 0; k < K; ++k) {
        SG_CHECK_ARG(d->elem_offsets[k] <= d->elem_offsets[k + 1], "logup: elem offsets");
        SG_CHECK_ARG(d->mult_term_offsets[k] <= d->mult_term_offsets[k + 1], "logup: mult offsets");
    }
    const uint32_t ne = d->elem_offsets[K], nmt = d->mult_term_offsets[K];
    for (uint32_t e = 0; e < ne; ++e) {
        SG_CHECK_ARG(d->term_offsets[e] <= d->term_offsets[e + 1], "logup: term offsets");
        SG_CHECK_ARG(d->elem_alpha_idx[e] < n_alpha, "logup: alpha power index out of range");
    }
    const uint32_t nt = ne ? d->term_offsets[ne] : 0;
    for (uint32_t q = 0; q < nt; ++q) SG_CHECK_ARG(d->term_cols[q] < m, "logup: fingerprint term column out of range");
    for (uint32_t q = 0; q < nmt; ++q) SG_CHECK_ARG(d->mult_term_cols[q] < m, "logup: multiplicity column out of range");
    return SG_OK;
}

}  // namespace sg

using namespace sg;

extern "C" {

int sg_eval_constraints(sg_ctx* c, void* stream, const sg_device_program* prog, const uint64_t* rap, uint32_t n_rap,
                        const uint64_t* alpha, uint32_t n_alpha, const uint64_t table_offset[3],
                        const uint64_t* d_main, uint64_t m, const uint64_t* d_aux, uint64_t a, uint64_t rows,
                        uint64_t next_step, const sg_composition* comp, uint64_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && prog && table_offset, "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(rows >= 1 && next_step < rows, "bad row count / frame step");
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t nn = prog->num_nodes, nr = prog->num_roots;
    const uint32_t nbs = prog->num_base_slots, nes = prog->num_ext_slots;
    // Validate the blob on the host: every slot, table index, column and frame
    // offset must be in range, so the walk never reads out of bounds. Count
    // the main-trace operands a row reads, for the layout choice below.
    uint64_t main_reads = 0;
    auto is_main_operand = [](uint32_t enc) {
        return (enc >> OPK_SHIFT) == OPK_VAR && !(enc & VAR_AUX_BIT) ? 1u : 0u;
    };
    auto is_base_operand = [&](uint32_t enc) {
        const uint32_t k = enc >> OPK_SHIFT;
        return k == OPK_BASE_SLOT || k == OPK_BASE_CONST || is_main_operand(enc);
    };
    for (uint32_t i = 0; i < nn; ++i) {
        const uint32_t* nd = prog->nodes + 4 * i;
        const uint32_t op = nd[0], slot = nd[3] & RES_SLOT_MASK;
        const bool rx = (nd[3] & RES_EXT_BIT) != 0;
        SG_CHECK_ARG(op <= OP_EMBED, "unknown op tag");
        SG_CHECK_ARG(rx ? slot < nes : slot < nbs, "result slot out of range");
        // result dims: constants and main-trace reads are base; extension
        // constants, challenges, the offset, embeddings and aux reads are
        // extension; a base arithmetic node has base operands only
        const bool var_main = op == OP_VAR && ((nd[2] >> 16) & 1u);
        if (op == OP_CONST_BASE || var_main) SG_CHECK_ARG(!rx, "a base node with an extension result slot");
        if ((op == OP_VAR && !var_main) || op == OP_CONST_EXT || op == OP_RAP_CHALLENGE || op == OP_ALPHA_POW ||
            op == OP_TABLE_OFFSET || op == OP_EMBED)
            SG_CHECK_ARG(rx, "an extension node with a base result slot");
        if (!rx && op >= OP_ADD && op <= OP_NEG)
            SG_CHECK_ARG(is_base_operand(nd[1]) && (op == OP_NEG || is_base_operand(nd[2])),
                         "a base node with an extension operand");
        auto ok_operand = [&](uint32_t enc) {
            const uint32_t k = enc >> OPK_SHIFT, p = enc & OPK_PAYLOAD_MASK;
            switch (k) {
                case OPK_BASE_SLOT: return p < nbs;
                case OPK_EXT_SLOT: return p < nes;
                case OPK_BASE_CONST: return p < prog->num_base_consts;
                case OPK_EXT_CONST: return p < prog->num_ext_consts;
                case OPK_RAP: return p < n_rap;
                case OPK_ALPHA: return p < n_alpha;
                case OPK_OFFSET: return true;
                case OPK_VAR:
                    return ((p & VAR_AUX_BIT) ? (p & VAR_COL_MASK) < a : (p & VAR_COL_MASK) < m) &&
                           (uint64_t)((p >> VAR_OFF_SHIFT) & 0xFFu) * next_step < rows && !(p & ~(VAR_AUX_BIT | (0xFFu << VAR_OFF_SHIFT) | VAR_COL_MASK));
                default: return false;
            }
        };
        if (op >= OP_ADD && op <= OP_MUL) SG_CHECK_ARG(ok_operand(nd[1]) && ok_operand(nd[2]), "operand out of range");
        if (op >= OP_ADD && op <= OP_EMBED) main_reads += is_main_operand(nd[1]);
        if (op >= OP_ADD && op <= OP_MUL) main_reads += is_main_operand(nd[2]);
        if (op == OP_NEG || op == OP_EMBED) SG_CHECK_ARG(ok_operand(nd[1]), "operand out of range");
        if (op == OP_VAR) {
            const uint32_t col = nd[1] & 0xFFFFu, off = (nd[2] >> 8) & 0xFFu;
            const bool main = ((nd[2] >> 16) & 1u) != 0;
            SG_CHECK_ARG(main ? col < m : col < a, "trace column out of range");
            SG_CHECK_ARG((uint64_t)off * next_step < rows, "frame offset wraps more than once");
        }
        if (op == OP_CONST_BASE) SG_CHECK_ARG(nd[1] < prog->num_base_consts, "constant index");
        if (op == OP_CONST_EXT) SG_CHECK_ARG(nd[1] < prog->num_ext_consts, "constant index");
        if (op == OP_RAP_CHALLENGE) SG_CHECK_ARG(nd[1] < n_rap, "challenge index");
        if (op == OP_ALPHA_POW) SG_CHECK_ARG(nd[1] < n_alpha, "alpha index");
    }
    const uint32_t hand = prog->hand_kernel ? prog->hand_roots : 0;
    const uint32_t hand_id = prog->hand_kernel & 0xFFu, hand_chips = prog->hand_kernel >> 8;
    if (prog->hand_kernel) {
        SG_CHECK_ARG(prog->node_roots && nr >= hand, "a hand kernel needs a streaming program");
        if (hand_id == SG_AIR_KECCAK)
            SG_CHECK_ARG(hand == KAIR_CONSTRAINTS && m == KAIR_WIDTH && !hand_chips, "not the KECCAK table's program");
        else if (hand_id == SG_AIR_SHIFT)
            SG_CHECK_ARG(hand == SH_CONSTRAINTS && m == SH_WIDTH && !hand_chips, "not the SHIFT table's program");
        else if (hand_id == SG_AIR_CPU)
            SG_CHECK_ARG(hand_chips < 16 && hand == cpu_air_constraints(hand_chips) &&
                             m == (hand_chips ? CPU_FULL_WIDTH : CPU_CORE_WIDTH),
                         "not the CPU table's program");
        else
            SG_CHECK_ARG(false, "unknown hand kernel");
    }
    // LogUp constraints evaluated from the table's descriptor: [lg_root, lg_root + lg_n)
    const sg_logup_desc* lg = prog->logup;
    const uint32_t lg_root = lg ? prog->logup_root : 0, lg_n = lg ? lg->num_committed + 1 : 0;
    if (lg) {
        SG_CHECK_ARG(prog->node_roots, "LogUp constraints from a descriptor need a streaming program");
        SG_TRY(check_logup_desc(lg, m, n_alpha));
        SG_CHECK_ARG(n_rap >= 1 && rap, "LogUp constraints need z = rap[0]");
        SG_CHECK_ARG(a >= lg_n && d_aux, "LogUp constraints need the committed and accumulated aux columns");
        SG_CHECK_ARG(lg_root >= hand && (uint64_t)lg_root + lg_n <= nr, "LogUp constraint indices out of range");
    }
    auto by_library = [&](uint32_t c) { return c < hand || (c >= lg_root && c - lg_root < lg_n); };
    if (prog->node_roots) {
        // streaming: every constraint completed by exactly one instruction
        // (those of a hand kernel or of the LogUp descriptor by none)
        std::vector<uint8_t> seen(nr, 0);
        for (uint32_t i = 0; i < nn; ++i) {
            const uint32_t c = prog->node_roots[i];
            if (c == NO_ROOT) continue;
            SG_CHECK_ARG(c < nr && !by_library(c) && !seen[c], "node_roots: constraint index out of range or repeated");
            seen[c] = 1;
        }
        for (uint32_t c = 0; c < nr; ++c)
            SG_CHECK_ARG(seen[c] || by_library(c), "node_roots: a constraint no instruction completes");
    } else {
        for (uint32_t r = 0; r < nr; ++r) {
            const uint32_t e = prog->roots[r];
            SG_CHECK_ARG((e & RES_EXT_BIT) ? (e & RES_SLOT_MASK) < nes : (e & RES_SLOT_MASK) < nbs, "root slot");
        }
    }
    if (comp) {
        SG_CHECK_ARG(comp->z_len >= 1 && comp->d_z_inv && comp->beta_trans, "composition inputs");
        for (uint32_t b = 0; b < comp->num_boundary; ++b)
            SG_CHECK_ARG(comp->b_is_aux[b] ? comp->b_col[b] < a : comp->b_col[b] < m, "boundary column");
    }
    // One device blob: nodes | roots | base consts | ext consts | rap | alpha | comp arrays.
    std::vector<uint64_t> blob;
    auto put = [&](const void* p, size_t bytes) {
        const size_t off = blob.size();
        blob.resize(off + (bytes + 7) / 8 + 1, 0);
        if (bytes) memcpy(blob.data() + off, p, bytes);
        return off;
    };
    const size_t o_nodes = put(prog->nodes, 16ull * nn);
    // `roots` is read only by the reference shape; a streaming program's
    // caller may pass fewer entries (or none), so nothing is copied from it
    const size_t o_roots = prog->node_roots ? put(nullptr, 0) : put(prog->roots, 4ull * nr);
    const size_t o_nroots = prog->node_roots ? put(prog->node_roots, 4ull * nn) : 0;
    const size_t o_bc = put(prog->base_consts, 8ull * prog->num_base_consts);
    const size_t o_ec = put(prog->ext_consts, 24ull * prog->num_ext_consts);
    const size_t o_rap = put(rap, 24ull * n_rap);
    const size_t o_al = put(alpha, 24ull * n_alpha);
    size_t o_lg[11] = {0};
    if (lg) {
        const uint32_t K = lg->num_interactions, ne = lg->elem_offsets[K], nt = ne ? lg->term_offsets[ne] : 0,
                       nmt = lg->mult_term_offsets[K];
        o_lg[0] = put(lg->bus_ids, 8ull * K);
        o_lg[1] = put(lg->elem_consts, 8ull * ne);
        o_lg[2] = put(lg->term_coefs, 8ull * nt);
        o_lg[3] = put(lg->mult_consts, 8ull * K);
        o_lg[4] = put(lg->mult_term_coefs, 8ull * nmt);
        o_lg[5] = put(lg->elem_offsets, 4ull * (K + 1));
        o_lg[6] = put(lg->elem_alpha_idx, 4ull * ne);
        o_lg[7] = put(lg->term_offsets, 4ull * (ne + 1));
        o_lg[8] = put(lg->term_cols, 4ull * nt);
        o_lg[9] = put(lg->mult_term_offsets, 4ull * (K + 1));
        o_lg[10] = put(lg->mult_term_cols, 4ull * nmt);
    }
    size_t o_beta = 0, o_bcol = 0, o_baux = 0, o_bval = 0, o_bbeta = 0;
    const uint32_t nb = comp ? comp->num_boundary : 0;
    if (comp) {
        o_beta = put(comp->beta_trans, 24ull * nr);
        o_bcol = put(comp->b_col, 8ull * nb);
        o_baux = put(comp->b_is_aux, 8ull * nb);
        o_bval = put(comp->b_value, 24ull * nb);
        o_bbeta = put(comp->b_beta, 24ull * nb);
    }
    // Shared-memory slot file when it fits (>= 32 threads per CTA), else global.
    const uint64_t per_thread = (uint64_t)nbs + 3ull * nes;
    int T = 128;
    while (T > 32 && per_thread * T * 8 > 160 * 1024) T -= 32;
    const bool use_smem = per_thread * T * 8 <= 160 * 1024;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t blocks = (rows + T - 1) / T;
    const uint64_t max_blocks = (uint64_t)sms * 16;
    if (blocks > max_blocks) blocks = max_blocks;
    uint64_t* d_blob = nullptr;
    uint64_t* d_scr = nullptr;
    const uint64_t bb = 8 * blob.size();
    const uint64_t sb = use_smem ? 0 : per_thread * blocks * T * 8;
    SG_TRY(dev_alloc(ctx, st, bb, (void**)&d_blob));
    int rc = SG_OK;
    if (!use_smem) rc = dev_alloc(ctx, st, sb, (void**)&d_scr);
    if (rc == SG_OK && cudaMemcpyAsync(d_blob, blob.data(), bb, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        set_error("constraints: program upload failed");
        rc = SG_ERR_CUDA;
    }
    if (rc == SG_OK) {
        Uni u{d_blob + o_bc, d_blob + o_ec, d_blob + o_rap, d_blob + o_al,
              fe3{table_offset[0], table_offset[1], table_offset[2]}};
        // A streaming walk reads the main LDE where each operand is used: a
        // column-major copy makes those reads coalesced (a warp's 32 rows are
        // one segment; row-major, each read moves a 32-byte sector for 8
        // bytes). The copy moves 2m words a row, so it pays once a row reads
        // at least m operands; skipped when the budget has no room for it.
        // The KECCAK kernel takes it too; the CPU and SHIFT tables' kernels
        // read their rows' columns nearly in order, so the rest of each
        // sector is still in L1 when it is needed, and measured faster
        // without the copy (with the copy's time: CPU 2^22 rows 24.2 ->
        // 20.5 ms, SHIFT 2^20 rows 3.53 -> 2.82 ms).
        uint64_t* d_cm = nullptr;
        const uint64_t cm_bytes = rows * m * 8;
        const bool hand_copy = hand && hand_id == SG_AIR_KECCAK;
        if (prog->node_roots && m >= CM_MIN_COLS && (main_reads >= m || hand_copy) && rows >= 32 &&
            rows / 32 <= 0x7FFFFFFFull && m / 32 < 65535) {
            if (dev_alloc(ctx, st, cm_bytes, (void**)&d_cm) == SG_OK) {
                k_to_columns<<<dim3((unsigned)((rows + 31) / 32), (unsigned)((m + 31) / 32)), dim3(32, 8), 0, st>>>(
                    d_main, rows, m, d_cm);
                rc = check_launch(ctx, "k_to_columns");
            } else {
                d_cm = nullptr;  // no room: the walk reads the row-major LDE
            }
        }
        Trace t{d_main, m, d_aux, a, rows, next_step, d_cm};
        Comp cp{};
        if (comp) {
            cp = Comp{d_blob + o_beta, comp->d_z_inv, comp->z_len, nb, d_blob + o_bcol, d_blob + o_baux,
                      d_blob + o_bval, d_blob + o_bbeta, comp->d_b_z_inv};
        }
        const size_t smem = use_smem ? per_thread * T * 8 : 0;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k_constraints, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const uint32_t* d_nroots = prog->node_roots ? (const uint32_t*)(d_blob + o_nroots) : nullptr;
        // the library's own constraint kernels first (a hand-written table
        // kernel, the LogUp descriptor's): per-row sums the walk starts from
        // (composition), or their values written directly (per constraint)
        uint64_t* d_extra = nullptr;
        const uint64_t extra_bytes = rows * 24;
        if (rc == SG_OK && comp && (hand || lg)) rc = dev_alloc(ctx, st, extra_bytes, (void**)&d_extra);
        if (rc == SG_OK && hand) {
            const uint64_t hb = (rows + 127) / 128, hcap = 148ull * 16;
            const unsigned grid = (unsigned)(hb < hcap ? hb : hcap);
            if (hand_id == SG_AIR_KECCAK) {
                k_keccak_constraints<<<grid, 128, 0, st>>>(d_cm, d_main, rows, next_step, keccak_consts(),
                                                           d_blob + o_beta, comp ? 0 : 1, comp ? d_extra : d_out);
                rc = check_launch(ctx, "k_keccak_constraints");
            } else if (hand_id == SG_AIR_SHIFT) {
                k_shift_constraints<<<grid, 128, 0, st>>>(d_cm, d_main, rows, next_step, d_blob + o_beta,
                                                          comp ? 0 : 1, comp ? d_extra : d_out);
                rc = check_launch(ctx, "k_shift_constraints");
            } else {
                k_cpu_constraints<<<grid, 128, 0, st>>>(d_cm, d_main, m, rows, next_step, hand_chips,
                                                        d_blob + o_beta, comp ? 0 : 1, comp ? d_extra : d_out);
                rc = check_launch(ctx, "k_cpu_constraints");
            }
        }
        if (rc == SG_OK && lg) {
            const uint64_t* b = d_blob;
            LogupDev dv{b + o_lg[0], b + o_lg[1], b + o_lg[2], b + o_lg[3], b + o_lg[4],
                        (const uint32_t*)(b + o_lg[5]), (const uint32_t*)(b + o_lg[6]), (const uint32_t*)(b + o_lg[7]),
                        (const uint32_t*)(b + o_lg[8]), (const uint32_t*)(b + o_lg[9]), (const uint32_t*)(b + o_lg[10]),
                        lg->num_interactions, lg->num_committed};
            const uint64_t lb = (rows + 127) / 128, lcap = 148ull * 16;
            k_logup_constraints<<<(unsigned)(lb < lcap ? lb : lcap), 128, 0, st>>>(
                t, dv, fe3{rap[0], rap[1], rap[2]}, d_blob + o_al, u.offset, d_blob + o_beta, lg_root, comp ? 0 : 1,
                hand ? 1 : 0, comp ? d_extra : d_out);
            rc = check_launch(ctx, "k_logup_constraints");
        }
        if (rc == SG_OK) {
            k_constraints<<<(unsigned)blocks, T, smem, st>>>((const uint4*)(d_blob + o_nodes), nn,
                                                             (const uint32_t*)(d_blob + o_roots), nr, d_nroots, nbs,
                                                             nes, u, t, cp, comp ? 0 : 1, d_out,
                                                             use_smem ? nullptr : d_scr, d_extra);
            rc = check_launch(ctx, "k_constraints");
        }
        if (rc == SG_OK && cudaStreamSynchronize(st) != cudaSuccess) {
            set_error("constraints: execution failed");
            rc = SG_ERR_CUDA;
        }
        if (d_cm) dev_free(ctx, st, d_cm, cm_bytes);
        if (d_extra) dev_free(ctx, st, d_extra, extra_bytes);
    }
    if (d_scr) dev_free(ctx, st, d_scr, sb);
    dev_free(ctx, st, d_blob, bb);
    return rc;
}

int sg_decompose_d2(sg_ctx* c, void* stream, const uint64_t* d_h, uint64_t lde_rows, const uint64_t* d_inv_2x,
                    uint64_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx, "null context");
    SG_ENTER(ctx);
    SG_CHECK_ARG(lde_rows % 2 == 0, "even LDE size required");
    const uint64_t n = lde_rows / 2;
    if (n == 0) return SG_OK;
    const uint64_t two_inv = (GL_P + 1) / 2;
    k_decompose_d2<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_h, d_inv_2x, two_inv, n, d_out);
    return check_launch(ctx, "k_decompose_d2");
}

}  // extern "C"
