// The RV64 CPU and SHIFT tables' layouts, and their constraints as
// hand-written kernels.
//
// The CPU table (lambda_vm_b200/rv64_air.py CpuAir) has 200 or 234 columns
// and ~300 base-field constraints (one-hot selectors, operand reads from the
// register file carried in the row, 32-bit limb arithmetic, the register-file
// transitions). This kernel evaluates them directly, one thread per LDE row,
// and folds them into the composition with the CpuAir emission order's
// constraint indices, so its sum equals the constraint walk's exactly. The
// chips the proof carries (bitwise, shift, memory, keccak) decide which
// constraint blocks exist, as in CpuAir. The LogUp constraints come from the
// table's descriptor (k_logup_constraints).
#pragma once

#include <stdint.h>

#include "gl.cuh"
#include "keccak_air.cuh"

namespace sg {

// Column layout of the CPU table: the core columns and the register file
// (CPU_CORE_WIDTH), then the chips' columns. Selector of op id i (1-based,
// rv64.py OPS order, 18 = the keccak ecall): CPU_SEL0 + i - 1.
constexpr uint32_t CPU_PC = 0, CPU_STEP = 1, CPU_CLK = 2, CPU_SEL0 = 3, CPU_RD0 = 21, CPU_RS10 = 53, CPU_RS20 = 85,
                   CPU_IMM_LO = 117, CPU_IMM_HI = 118, CPU_IMM_F = 119, CPU_A_LO = 120, CPU_A_HI = 121,
                   CPU_B_LO = 122, CPU_B_HI = 123, CPU_R_LO = 124, CPU_R_HI = 125, CPU_R16 = 126, CPU_C0 = 130,
                   CPU_C1 = 131, CPU_INV_LO = 132, CPU_INV_HI = 133, CPU_E_LO = 134, CPU_E_HI = 135, CPU_NE = 136,
                   CPU_BR = 137, CPU_X0 = 138, CPU_CORE_WIDTH = 200, CPU_AB0 = 200, CPU_BB0 = 208, CPU_RB0 = 216,
                   CPU_MA = 224, CPU_MW0 = 225, CPU_MW1 = 226, CPU_MV_LO = 227, CPU_MV_HI = 228, CPU_MT = 229,
                   CPU_MD0 = 230, CPU_MD1 = 231, CPU_NV_LO = 232, CPU_NV_HI = 233, CPU_FULL_WIDTH = 234;
enum CpuOp : uint32_t {
    OPC_ADD = 1, OPC_SUB, OPC_ADDI, OPC_LUI, OPC_BEQ, OPC_BNE, OPC_ECALL, OPC_XOR, OPC_OR, OPC_AND, OPC_XORI,
    OPC_ORI, OPC_ANDI, OPC_SLLI, OPC_SRLI, OPC_LD, OPC_SD, OPC_KECCAK
};
constexpr uint32_t CHIP_BITWISE = 1, CHIP_SHIFT = 2, CHIP_MEMORY = 4, CHIP_KECCAK = 8;

// The number of base constraints CpuAir emits for a chip set.
__host__ __device__ constexpr uint32_t cpu_air_constraints(uint32_t chips) {
    const bool bw = chips & CHIP_BITWISE, sh = chips & CHIP_SHIFT, mem = chips & CHIP_MEMORY,
               kc = chips & CHIP_KECCAK;
    const uint32_t absent = (bw ? 0 : 6) + (sh ? 0 : 2) + (mem ? 0 : 2) + ((kc && mem) ? 0 : 1);
    return 117 + 4 + absent + 30 + (bw ? 6 : 0) + (mem ? 12 : 0) + 64 + 65;
}

struct CRow {
    const uint64_t* cm;
    const uint64_t* rm;
    uint64_t rows, width, row, rn;
    __device__ __forceinline__ uint64_t at(uint64_t r, uint32_t col) const {
        return cm ? cm[(uint64_t)col * rows + r] : rm[r * width + col];
    }
    __device__ __forceinline__ uint64_t M(uint32_t col) const { return at(row, col); }
    __device__ __forceinline__ uint64_t N(uint32_t col) const { return at(rn, col); }
    __device__ __forceinline__ uint64_t sel(uint32_t op) const { return M(CPU_SEL0 + op - 1); }
};

__device__ __forceinline__ uint32_t cpu_xlo(uint32_t k) { return CPU_X0 + 2 * (k - 1); }

static __global__ void k_cpu_constraints(const uint64_t* __restrict__ cm, const uint64_t* __restrict__ rm,
                                         uint64_t width, uint64_t rows, uint64_t next_step, uint32_t chips,
                                         const uint64_t* __restrict__ beta, int mode, uint64_t* __restrict__ out) {
    const uint64_t K32 = 1ull << 32, K16 = 1ull << 16;
    for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows;
         row += (uint64_t)gridDim.x * blockDim.x) {
        const CRow w{cm, rm, rows, width, row, row + next_step >= rows ? row + next_step - rows : row + next_step};
        KSink s{beta, mode, out, rows, row, gl::wzero3(), 0};
        const uint64_t step = w.M(CPU_STEP), c0 = w.M(CPU_C0), c1 = w.M(CPU_C1);
        // one-hot selections and booleans
        s.put(kbool(step));
        s.put(kbool(c0));
        s.put(kbool(c1));
        for (uint32_t i = 0; i < 18; ++i) s.put(kbool(w.M(CPU_SEL0 + i)));
        for (uint32_t g = CPU_RD0; g < CPU_RS20 + 32; g += 32)
            for (uint32_t k = 0; k < 32; ++k) s.put(kbool(w.M(g + k)));
        {
            uint64_t t = 0;
            for (uint32_t i = 0; i < 18; ++i) t = gl::add(t, w.M(CPU_SEL0 + i));
            s.put(gl::sub(t, 1));
        }
        for (uint32_t g = CPU_RD0; g < CPU_RS20 + 32; g += 32) {
            uint64_t t = 0;
            for (uint32_t k = 0; k < 32; ++k) t = gl::add(t, w.M(g + k));
            s.put(gl::sub(t, 1));
        }
        // an instruction whose chip the proof does not carry cannot occur
        if (!(chips & CHIP_BITWISE))
            for (uint32_t op = OPC_XOR; op <= OPC_ANDI; ++op) s.put(w.sel(op));
        if (!(chips & CHIP_SHIFT)) s.put(w.sel(OPC_SLLI)), s.put(w.sel(OPC_SRLI));
        if (!(chips & CHIP_MEMORY)) s.put(w.sel(OPC_LD)), s.put(w.sel(OPC_SD));
        if (!(chips & CHIP_KECCAK) || !(chips & CHIP_MEMORY)) s.put(w.sel(OPC_KECCAK));
        // operand reads: a = x[rs1], b = x[rs2]
        for (uint32_t op2 = 0; op2 < 2; ++op2)
            for (uint32_t limb = 0; limb < 2; ++limb) {
                const uint32_t base = op2 ? CPU_RS20 : CPU_RS10;
                gl::wacc t = gl::wzero();  // the 31 products summed unreduced
                for (uint32_t k = 1; k < 32; ++k) gl::wmac(t, w.M(base + k), w.M(cpu_xlo(k) + limb));
                s.put(gl::sub(w.M((base == CPU_RS10 ? CPU_A_LO : CPU_B_LO) + limb), gl::wreduce(t)));
            }
        const uint64_t rl = w.M(CPU_R_LO), rh = w.M(CPU_R_HI), al = w.M(CPU_A_LO), ah = w.M(CPU_A_HI),
                       bl = w.M(CPU_B_LO), bh = w.M(CPU_B_HI), il = w.M(CPU_IMM_LO), ih = w.M(CPU_IMM_HI);
        // the written value in 16-bit pieces
        s.put(gl::sub(rl, gl::add(w.M(CPU_R16), gl::mul(K16, w.M(CPU_R16 + 1)))));
        s.put(gl::sub(rh, gl::add(w.M(CPU_R16 + 2), gl::mul(K16, w.M(CPU_R16 + 3)))));
        // add / addi, sub, lui
        const uint64_t s_add = w.sel(OPC_ADD), s_addi = w.sel(OPC_ADDI), s_sub = w.sel(OPC_SUB), s_lui = w.sel(OPC_LUI);
        const uint64_t c0k = gl::mul(c0, K32), c1k = gl::mul(c1, K32);
        s.put(gl::mul(s_add, gl::sub(gl::add(rl, c0k), gl::add(al, bl))));
        s.put(gl::mul(s_add, gl::sub(gl::add(rh, c1k), gl::add(gl::add(ah, bh), c0))));
        s.put(gl::mul(s_addi, gl::sub(gl::add(rl, c0k), gl::add(al, il))));
        s.put(gl::mul(s_addi, gl::sub(gl::add(rh, c1k), gl::add(gl::add(ah, ih), c0))));
        s.put(gl::mul(s_sub, gl::sub(gl::add(rl, bl), gl::add(al, c0k))));
        s.put(gl::mul(s_sub, gl::sub(gl::add(gl::add(rh, bh), c0), gl::add(ah, c1k))));
        s.put(gl::mul(s_lui, gl::sub(rl, il)));
        s.put(gl::mul(s_lui, gl::sub(rh, ih)));
        // no value for branches, ecalls and stores; carries only where an addition uses them
        const uint64_t s_beq = w.sel(OPC_BEQ), s_bne = w.sel(OPC_BNE), s_ecall = w.sel(OPC_ECALL),
                       s_kec = w.sel(OPC_KECCAK), s_ld = w.sel(OPC_LD), s_sd = w.sel(OPC_SD);
        const uint64_t nores = gl::add(gl::add(gl::add(gl::add(s_beq, s_bne), s_ecall), s_kec), s_sd);
        s.put(gl::mul(nores, rl));
        s.put(gl::mul(nores, rh));
        const uint64_t nocarry =
            gl::sub(1, gl::add(gl::add(gl::add(gl::add(s_add, s_addi), s_sub), s_ld), s_sd));
        s.put(gl::mul(nocarry, c0));
        s.put(gl::mul(nocarry, c1));
        // branch witnesses
        const uint64_t branch = gl::add(s_beq, s_bne);
        const uint64_t el = w.M(CPU_E_LO), eh = w.M(CPU_E_HI);
        for (uint32_t limb = 0; limb < 2; ++limb) {
            const uint64_t d = limb ? gl::sub(ah, bh) : gl::sub(al, bl);
            const uint64_t e = limb ? eh : el, inv = w.M(limb ? CPU_INV_HI : CPU_INV_LO);
            s.put(gl::mul(branch, gl::sub(e, gl::mul(d, inv))));
            s.put(gl::mul(branch, gl::mul(d, gl::sub(1, e))));
            s.put(gl::mul(gl::sub(1, branch), e));
        }
        const uint64_t ne = w.M(CPU_NE), br = w.M(CPU_BR);
        s.put(gl::sub(ne, gl::sub(gl::add(el, eh), gl::mul(el, eh))));
        s.put(gl::sub(br, gl::add(gl::mul(s_beq, gl::sub(1, ne)), gl::mul(s_bne, ne))));
        // ecalls: exit with a7 = 93, keccak with a7 = 2^64 - 2
        const uint64_t x17l = w.M(cpu_xlo(17)), x17h = w.M(cpu_xlo(17) + 1);
        s.put(gl::mul(s_ecall, gl::sub(x17l, 93)));
        s.put(gl::mul(s_ecall, x17h));
        s.put(gl::mul(s_kec, gl::sub(x17l, 0xFFFFFFFEull)));
        s.put(gl::mul(s_kec, gl::sub(x17h, 0xFFFFFFFFull)));
        if (chips & CHIP_BITWISE) {
            const uint64_t sreg = gl::add(gl::add(w.sel(OPC_XOR), w.sel(OPC_OR)), w.sel(OPC_AND));
            const uint64_t simm = gl::add(gl::add(w.sel(OPC_XORI), w.sel(OPC_ORI)), w.sel(OPC_ANDI));
            const uint64_t sbit = gl::add(sreg, simm);
            for (uint32_t limb = 0; limb < 2; ++limb) {
                auto bytes = [&](uint32_t first) {
                    uint64_t t = 0;
                    for (uint32_t i = 0; i < 4; ++i)
                        t = gl::add(t, gl::mul(1ull << (8 * i), w.M(first + i + 4 * limb)));
                    return t;
                };
                const uint64_t a_ = limb ? ah : al, b_ = limb ? bh : bl, i_ = limb ? ih : il, r_ = limb ? rh : rl;
                s.put(gl::mul(sbit, gl::sub(a_, bytes(CPU_AB0))));
                const uint64_t ob = bytes(CPU_BB0);
                s.put(gl::add(gl::mul(sreg, gl::sub(b_, ob)), gl::mul(simm, gl::sub(i_, ob))));
                s.put(gl::mul(sbit, gl::sub(r_, bytes(CPU_RB0))));
            }
        }
        if (chips & CHIP_MEMORY) {
            const uint64_t smem = gl::add(s_ld, s_sd), saddr = gl::add(smem, s_kec), ma = w.M(CPU_MA);
            s.put(gl::mul(smem, gl::sub(gl::add(ma, c0k), gl::add(al, il))));
            s.put(gl::mul(smem, gl::sub(c1k, gl::add(gl::add(ah, ih), c0))));
            s.put(gl::mul(s_kec, gl::sub(ma, w.M(cpu_xlo(10)))));
            s.put(gl::mul(s_kec, w.M(cpu_xlo(10) + 1)));
            s.put(gl::mul(saddr, gl::sub(ma, gl::add(gl::mul(8, w.M(CPU_MW0)), gl::mul(1ull << 19, w.M(CPU_MW1))))));
            const uint64_t gap = gl::sub(gl::sub(w.M(CPU_CLK), w.M(CPU_MT)), 1);
            s.put(gl::mul(smem, gl::sub(gap, gl::add(w.M(CPU_MD0), gl::mul(K16, w.M(CPU_MD1))))));
            for (uint32_t limb = 0; limb < 2; ++limb) {
                const uint64_t nv = w.M(limb ? CPU_NV_HI : CPU_NV_LO), mv = w.M(limb ? CPU_MV_HI : CPU_MV_LO);
                s.put(gl::mul(s_ld, gl::sub(nv, mv)));
                s.put(gl::mul(s_sd, gl::sub(nv, limb ? bh : bl)));
                s.put(gl::mul(s_ld, gl::sub(limb ? rh : rl, mv)));
            }
        }
        // transitions: next pc, timestamp and register file
        const uint64_t adv = gl::add(gl::mul(4, gl::sub(1, s_ecall)), gl::mul(br, gl::sub(w.M(CPU_IMM_F), 4)));
        s.put(gl::mul(step, gl::sub(w.N(CPU_PC), gl::add(w.M(CPU_PC), adv))));
        s.put(gl::mul(step, gl::sub(w.N(CPU_CLK), gl::add(w.M(CPU_CLK), 1))));
        for (uint32_t k = 1; k < 32; ++k) {
            const uint64_t rdk = w.M(CPU_RD0 + k);
            for (uint32_t limb = 0; limb < 2; ++limb) {
                const uint32_t col = cpu_xlo(k) + limb;
                const uint64_t x = w.M(col);
                const uint64_t upd = gl::mul(rdk, gl::sub(limb ? rh : rl, x));
                s.put(gl::mul(step, gl::sub(w.N(col), gl::add(x, upd))));
            }
        }
        // the END row: an exit ecall, followed by the initial state
        const uint64_t nstep = gl::sub(1, step);
        s.put(gl::mul(nstep, gl::sub(1, s_ecall)));
        s.put(gl::mul(nstep, w.N(CPU_PC)));
        s.put(gl::mul(nstep, gl::sub(w.N(CPU_CLK), 1)));
        for (uint32_t k = 1; k < 32; ++k) {
            s.put(gl::mul(nstep, w.N(cpu_xlo(k))));
            s.put(gl::mul(nstep, w.N(cpu_xlo(k) + 1)));
        }
        if (mode == 0) {
            uint64_t* o = out + 3 * row;
            const gl::fe3 sum = s.total();
            o[0] = sum.c0, o[1] = sum.c1, o[2] = sum.c2;
        }
    }
}

// The SHIFT table (rv64_air.py ShiftAir): DIR, the operand's bits, one-hot
// s = k mod 8 and q = k div 8, the operand shifted by s bits, the result's
// limbs, the multiplicity. Its 149 base constraints in ShiftAir's order.
constexpr uint32_t SH_DIR = 0, SH_AB = 1, SH_S = 65, SH_Q = 73, SH_TB = 81, SH_R_LO = 145, SH_R_HI = 146,
                   SH_WIDTH = 148, SH_CONSTRAINTS = 149;

static __global__ void k_shift_constraints(const uint64_t* __restrict__ cm, const uint64_t* __restrict__ rm,
                                           uint64_t rows, uint64_t next_step, const uint64_t* __restrict__ beta,
                                           int mode, uint64_t* __restrict__ out) {
    for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows;
         row += (uint64_t)gridDim.x * blockDim.x) {
        const CRow w{cm, rm, rows, SH_WIDTH, row, row};
        KSink s{beta, mode, out, rows, row, gl::wzero3(), 0};
        const uint64_t d = w.M(SH_DIR), nd = gl::sub(1, d);
        s.put(kbool(d));
        for (uint32_t i = 0; i < 64; ++i) s.put(kbool(w.M(SH_AB + i)));
        for (uint32_t i = 0; i < 8; ++i) s.put(kbool(w.M(SH_S + i)));
        for (uint32_t i = 0; i < 8; ++i) s.put(kbool(w.M(SH_Q + i)));
        uint64_t ts = 0, tq = 0;
        for (uint32_t i = 0; i < 8; ++i) ts = gl::add(ts, w.M(SH_S + i)), tq = gl::add(tq, w.M(SH_Q + i));
        s.put(gl::sub(ts, 1));
        s.put(gl::sub(tq, 1));
        // TB_j = sum_s S_s (nd a[j - s] + d a[j + s]), bits past either end
        // zero, evaluated as nd (sum_s S_s a[j - s]) + d (sum_s S_s a[j + s])
        // with both sums kept unreduced (the same polynomial)
        uint64_t sv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) sv[k] = w.M(SH_S + k);
        for (int j = 0; j < 64; ++j) {
            gl::wacc lo = gl::wzero(), hi = gl::wzero();
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (j - k >= 0) gl::wmac(lo, sv[k], w.M(SH_AB + j - k));
                if (j + k < 64) gl::wmac(hi, sv[k], w.M(SH_AB + j + k));
            }
            const uint64_t t = gl::add(gl::mul(nd, gl::wreduce(lo)), gl::mul(d, gl::wreduce(hi)));
            s.put(gl::sub(w.M(SH_TB + j), t));
        }
        // the result moves TB by whole bytes: byte k = sum_q Q_q (nd tB[k - q] + d tB[k + q])
        uint64_t tB[8];
        for (int i = 0; i < 8; ++i) {
            uint64_t t = 0;
            for (int j = 7; j >= 0; --j) t = gl::add(gl::add(t, t), w.M(SH_TB + 8 * i + j));
            tB[i] = t;
        }
        uint64_t qv[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) qv[q] = w.M(SH_Q + q);
        for (int limb = 0; limb < 2; ++limb) {
            uint64_t acc = 0;
            for (int k = 4 * limb + 3; k >= 4 * limb; --k) {
                gl::wacc lo = gl::wzero(), hi = gl::wzero();
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (k - q >= 0) gl::wmac(lo, qv[q], tB[k - q]);
                    if (k + q < 8) gl::wmac(hi, qv[q], tB[k + q]);
                }
                const uint64_t t = gl::add(gl::mul(nd, gl::wreduce(lo)), gl::mul(d, gl::wreduce(hi)));
                acc = gl::add(gl::mul(acc, 256), t);
            }
            s.put(gl::sub(w.M(limb ? SH_R_HI : SH_R_LO), acc));
        }
        if (mode == 0) {
            uint64_t* o = out + 3 * row;
            const gl::fe3 sum = s.total();
            o[0] = sum.c0, o[1] = sum.c1, o[2] = sum.c2;
        }
    }
}

}  // namespace sg
