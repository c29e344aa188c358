// RV64 front-end on the host: execute a guest of the supported RV64I subset
// and write the CPU table its proof needs, in one pass.
//
// The same machine and the same table as lambda_vm_b200/rv64.py (execute)
// and rv64_air.py (CpuAir.trace), which the tests compare this against: ADD,
// SUB, ADDI, LUI, BEQ, BNE and ECALL-exit (a7 = 93) on 64-bit registers with
// x0 hard-wired to zero (executor/src/vm semantics for these opcodes). One
// table row per executed instruction, padded to n rows by repeating the
// halting ECALL; the last row carries STEP = 0. Writing the 188-column rows as
// the machine runs keeps the whole front-end at memory speed on the host.
#include <string.h>

#include <vector>

#include "common.cuh"

namespace {

constexpr uint64_t P = 0xFFFFFFFF00000001ULL;
enum Op { ADD = 1, SUB, ADDI, LUI, BEQ, BNE, ECALL };  // the ROM tuple's opcode ids
// Column layout of the CPU table (rv64_air.py).
constexpr int PC = 0, STEP = 1, SEL0 = 2, RD0 = 9, RS10 = 41, RS20 = 73, IMM_LO = 105, IMM_HI = 106, IMM_F = 107,
              A_LO = 108, A_HI = 109, B_LO = 110, B_HI = 111, R_LO = 112, R_HI = 113, R16 = 114, C0 = 118, C1 = 119,
              INV_LO = 120, INV_HI = 121, E_LO = 122, E_HI = 123, NE = 124, BR = 125, X0 = 126;
static_assert(X0 + 62 == SG_RV64_CPU_WIDTH, "CPU table width");

struct Ins {
    int op, rd, rs1, rs2;
    int64_t imm;
};

uint32_t bits(uint32_t x, int hi, int lo) { return (x >> lo) & ((1u << (hi - lo + 1)) - 1); }
int64_t sext(uint64_t x, int b) {
    x &= (1ULL << b) - 1;
    return (x >> (b - 1)) ? (int64_t)x - (int64_t)(1ULL << b) : (int64_t)x;
}

bool decode(uint32_t w, Ins* o) {
    const uint32_t opc = w & 0x7F, rd = bits(w, 11, 7), f3 = bits(w, 14, 12), rs1 = bits(w, 19, 15),
                   rs2 = bits(w, 24, 20), f7 = bits(w, 31, 25);
    *o = Ins{0, (int)rd, (int)rs1, (int)rs2, 0};
    if (opc == 0x33 && f3 == 0 && (f7 == 0 || f7 == 0x20)) {
        o->op = f7 ? SUB : ADD;
    } else if (opc == 0x13 && f3 == 0) {
        *o = Ins{ADDI, (int)rd, (int)rs1, 0, sext(w >> 20, 12)};
    } else if (opc == 0x37) {
        *o = Ins{LUI, (int)rd, 0, 0, sext(w >> 12, 20) * 4096};
    } else if (opc == 0x63 && (f3 == 0 || f3 == 1)) {
        const uint32_t imm = (bits(w, 31, 31) << 12) | (bits(w, 7, 7) << 11) | (bits(w, 30, 25) << 5) | (bits(w, 11, 8) << 1);
        *o = Ins{f3 ? BNE : BEQ, 0, (int)rs1, (int)rs2, sext(imm, 13)};
    } else if (w == 0x00000073) {
        *o = Ins{ECALL, 0, 0, 0, 0};
    } else {
        return false;
    }
    return true;
}

}  // namespace

using namespace sg;

extern "C" int sg_rv64_trace(const uint32_t* words, uint32_t nwords, uint64_t max_steps, uint64_t n_rows,
                             uint64_t* trace_out, uint64_t* counts_out, uint64_t* a0_out, uint64_t* cycles_out) {
    SG_CHECK_ARG(words && nwords && cycles_out && a0_out, "null argument");
    SG_CHECK_ARG(!trace_out || (n_rows >= 2 && (n_rows & (n_rows - 1)) == 0), "n_rows must be a power of two >= 2");
    std::vector<Ins> prog(nwords);
    for (uint32_t i = 0; i < nwords; ++i) SG_CHECK_ARG(decode(words[i], &prog[i]), "unsupported instruction word");
    if (counts_out) memset(counts_out, 0, nwords * sizeof(uint64_t));
    uint64_t x[32] = {0};
    uint64_t pc = 0, t = 0;
    const uint64_t W = SG_RV64_CPU_WIDTH;
    auto row_of = [&](uint64_t r) { return trace_out + r * W; };
    bool halted = false;
    uint64_t halt_row = 0;
    while (!halted) {
        SG_CHECK_ARG(t < max_steps, "the program did not halt within max_steps");
        SG_CHECK_ARG(pc % 4 == 0 && pc / 4 < nwords, "pc outside the program");
        const Ins& in = prog[pc / 4];
        const uint64_t a = x[in.rs1], b = x[in.rs2];
        uint64_t r = 0, npc = pc + 4;
        switch (in.op) {
            case ADD: r = a + b; break;
            case SUB: r = a - b; break;
            case ADDI: r = a + (uint64_t)in.imm; break;
            case LUI: r = (uint64_t)in.imm; break;
            case BEQ: npc = a == b ? pc + (uint64_t)in.imm : pc + 4; break;
            case BNE: npc = a != b ? pc + (uint64_t)in.imm : pc + 4; break;
            case ECALL:
                SG_CHECK_ARG(x[17] == 93, "only the exit ecall (a7 = 93) is supported");
                halted = true;
                npc = pc;
                break;
        }
        if (trace_out) {
            SG_CHECK_ARG(t < n_rows, "the execution does not fit n_rows");
            uint64_t* row = row_of(t);
            memset(row, 0, W * 8);
            row[PC] = pc;
            row[STEP] = 1;
            row[SEL0 + in.op - 1] = 1;
            row[RD0 + in.rd] = 1;
            row[RS10 + in.rs1] = 1;
            row[RS20 + in.rs2] = 1;
            const uint64_t iu = (uint64_t)in.imm;
            row[IMM_LO] = iu & 0xFFFFFFFFULL;
            row[IMM_HI] = iu >> 32;
            row[IMM_F] = in.imm < 0 ? P - (uint64_t)(-in.imm) : iu;
            row[A_LO] = a & 0xFFFFFFFFULL, row[A_HI] = a >> 32;
            row[B_LO] = b & 0xFFFFFFFFULL, row[B_HI] = b >> 32;
            row[R_LO] = r & 0xFFFFFFFFULL, row[R_HI] = r >> 32;
            for (int j = 0; j < 4; ++j) row[R16 + j] = (r >> (16 * j)) & 0xFFFF;
            if (in.op == ADD || in.op == ADDI) {
                const uint64_t o = in.op == ADD ? b : iu;
                const uint64_t c0 = ((a & 0xFFFFFFFFULL) + (o & 0xFFFFFFFFULL)) >> 32;
                row[C0] = c0;
                row[C1] = ((a >> 32) + (o >> 32) + c0) >> 32;
            } else if (in.op == SUB) {
                const uint64_t b0 = (a & 0xFFFFFFFFULL) < (b & 0xFFFFFFFFULL);
                row[C0] = b0;
                row[C1] = (a >> 32) < (b >> 32) + b0;
            }
            if (in.op == BEQ || in.op == BNE) {
                const uint64_t dl = ((a & 0xFFFFFFFFULL) + P - (b & 0xFFFFFFFFULL)) % P;
                const uint64_t dh = ((a >> 32) + P - (b >> 32)) % P;
                row[INV_LO] = dl ? sg_host_gl_inv(dl) : 0;
                row[INV_HI] = dh ? sg_host_gl_inv(dh) : 0;
                row[E_LO] = dl != 0, row[E_HI] = dh != 0;
                const uint64_t ne = row[E_LO] | row[E_HI];
                row[NE] = ne;
                row[BR] = in.op == BNE ? ne : 1 - ne;
            }
            for (int k = 1; k < 32; ++k) {
                row[X0 + 2 * (k - 1)] = x[k] & 0xFFFFFFFFULL;
                row[X0 + 2 * (k - 1) + 1] = x[k] >> 32;
            }
        }
        if (counts_out) counts_out[pc / 4] += 1;
        if (in.rd && (in.op == ADD || in.op == SUB || in.op == ADDI || in.op == LUI)) x[in.rd] = r;
        halt_row = t;
        pc = npc;
        ++t;
    }
    *cycles_out = t;
    *a0_out = x[10];
    if (trace_out) {
        // the halting row repeats to fill the table; the last row ends the cycle
        for (uint64_t r = t; r < n_rows; ++r) memcpy(row_of(r), row_of(halt_row), W * 8);
        if (counts_out) counts_out[pc / 4] += n_rows - t;
        row_of(n_rows - 1)[STEP] = 0;
    }
    return SG_OK;
}
