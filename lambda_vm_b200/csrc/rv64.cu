// RV64 front-end on the host: execute a guest of the supported RV64I subset
// and write the CPU table its proof needs, in one pass, together with the
// events the chip tables are built from (shifts, the touched memory cells,
// the Keccak ecalls).
//
// The same machine and the same table as lambda_vm_b200/rv64.py (run) and
// rv64_air.py (CpuAir.trace), which the tests compare this against cell for
// cell: ADD, SUB, XOR, OR, AND, ADDI, XORI, ORI, ANDI, SLLI, SRLI, LUI, LD, SD,
// BEQ, BNE and ECALL (a7 = 93 exit, a7 = 2^64 - 2 keccak-f[1600] on the 25
// lanes at a0) on 64-bit registers with x0 hard-wired to zero (executor/src/vm
// semantics for these opcodes; the keccak ecall as
// executor/src/vm/instruction/execution.rs:649-670). Data memory starts
// zeroed; loads and stores are doublewords at 8-byte-aligned addresses below
// 2^32. One table row per executed instruction (row t has timestamp t + 1),
// padded to n rows by repeating the halting ECALL; the last row carries
// STEP = 0. Writing the rows as the machine runs keeps the front-end at
// memory speed on the host.
#include <string.h>
#include <sys/mman.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <algorithm>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "gl.cuh"
#include "keccak_air.cuh"

namespace {

constexpr uint64_t P = 0xFFFFFFFF00000001ULL;
constexpr uint64_t M32 = 0xFFFFFFFFULL;
constexpr uint64_t KECCAK_CALL = ~0ULL - 1;  // a7 of the keccak ecall
constexpr uint64_t EXIT_CALL = 93;
// the ROM tuple's opcode ids (rv64.py OPS order, from 1)
enum Op { ADD = 1, SUB, ADDI, LUI, BEQ, BNE, ECALL, XOR, OR, AND, XORI, ORI, ANDI, SLLI, SRLI, LD, SD };
// Column layout of the CPU table (rv64_air.py): the core columns and the
// register file (SG_RV64_CPU_CORE_WIDTH), then the chips' columns (to
// SG_RV64_CPU_WIDTH). SEL0 + op - 1 is an opcode's selector (KECCAK_OP: the
// keccak ecall's).
constexpr int KECCAK_OP = 18;
constexpr int PC = 0, STEP = 1, CLK = 2, SEL0 = 3, RD0 = 21, RS10 = 53, RS20 = 85, IMM_LO = 117, IMM_HI = 118,
              IMM_F = 119, A_LO = 120, A_HI = 121, B_LO = 122, B_HI = 123, R_LO = 124, R_HI = 125, R16 = 126, C0 = 130,
              C1 = 131, INV_LO = 132, INV_HI = 133, E_LO = 134, E_HI = 135, NE = 136, BR = 137, X0 = 138, AB0 = 200,
              BB0 = 208, RB0 = 216, MA = 224, MW0 = 225, MW1 = 226, MV_LO = 227, MV_HI = 228, MT = 229, MD0 = 230,
              MD1 = 231, NV_LO = 232, NV_HI = 233;
static_assert(X0 + 62 == SG_RV64_CPU_CORE_WIDTH && NV_HI + 1 == SG_RV64_CPU_WIDTH, "CPU table widths");

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
    if (opc == 0x33) {
        if (f3 == 0 && (f7 == 0 || f7 == 0x20)) o->op = f7 ? SUB : ADD;
        else if (f7 == 0 && f3 == 4) o->op = XOR;
        else if (f7 == 0 && f3 == 6) o->op = OR;
        else if (f7 == 0 && f3 == 7) o->op = AND;
        else return false;
    } else if (opc == 0x13) {
        if (f3 == 1 || f3 == 5) {
            if (bits(w, 31, 26) != 0) return false;
            *o = Ins{f3 == 1 ? SLLI : SRLI, (int)rd, (int)rs1, 0, (int64_t)bits(w, 25, 20)};
        } else {
            const int op = f3 == 0 ? ADDI : f3 == 4 ? XORI : f3 == 6 ? ORI : f3 == 7 ? ANDI : 0;
            if (!op) return false;
            *o = Ins{op, (int)rd, (int)rs1, 0, sext(w >> 20, 12)};
        }
    } else if (opc == 0x03 && f3 == 3) {
        *o = Ins{LD, (int)rd, (int)rs1, 0, sext(w >> 20, 12)};
    } else if (opc == 0x23 && f3 == 3) {
        *o = Ins{SD, 0, (int)rs1, (int)rs2, sext((f7 << 5) | rd, 12)};
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

uint64_t rotl(uint64_t v, int r) { return r ? (v << r) | (v >> (64 - r)) : v; }
void keccak_f(uint64_t a[25]) {
    const sg::KeccakTables& k = sg::keccak_tables();
    for (int ir = 0; ir < 24; ++ir) {
        uint64_t c[5], d[5], b[25];
        for (int x = 0; x < 5; ++x) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
        for (int x = 0; x < 5; ++x) d[x] = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(a[x + 5 * y] ^ d[x], k.rot[x + 5 * y]);
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= k.rc[ir];
    }
}

struct Cell {
    uint64_t value, stamp;  // stamp 0: never accessed
};

// Data memory: 8-byte cells in pages of 4096, allocated on first touch, the
// last page cached (a guest's accesses stay in a few pages at a time).
class Memory {
  public:
    Cell* at(uint64_t addr) {
        const uint64_t pg = addr >> 15;
        if (pg != last_pg_ || !last_) {
            auto& p = pages_[pg];
            if (!p) p.reset(new Cell[4096]());
            last_pg_ = pg, last_ = p.get();
        }
        return last_ + ((addr >> 3) & 4095);
    }
    // every accessed cell in ascending address order
    template <class F>
    void each_touched(F f) const {
        std::vector<uint64_t> pgs;
        for (const auto& kv : pages_) pgs.push_back(kv.first);
        std::sort(pgs.begin(), pgs.end());
        for (uint64_t pg : pgs) {
            const Cell* c = pages_.at(pg).get();
            for (uint64_t i = 0; i < 4096; ++i)
                if (c[i].stamp) f((pg << 15) | (i << 3), c[i]);
        }
    }

  private:
    std::unordered_map<uint64_t, std::unique_ptr<Cell[]>> pages_;
    uint64_t last_pg_ = ~0ull;
    Cell* last_ = nullptr;
};

// The CPU table's lookups, counted from the row records after the run, a
// slice of rows per host thread into thread-local histograms: RANGE (the
// written value's four 16-bit pieces on every row, the address pieces of
// memory and keccak rows, the timestamp-gap pieces of memory rows) and
// BITWISE (the eight byte pairs of a bitwise row, by kind).
void count_cpu_lookups(const uint64_t* rec, uint64_t T, uint64_t* range_counts, uint64_t* bitwise_counts) {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned nt = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>({hw ? hw : 1u, 16u, T / 65536 + 1}));
    const uint32_t RB = range_counts ? 65536 : 0, BB = bitwise_counts ? 3 * 65536 : 0;
    // one histogram block per thread (RANGE bins then BITWISE bins), each
    // zeroed by its own thread; then the blocks are summed bin slice by bin
    // slice, also one slice per thread
    std::unique_ptr<uint32_t[]> hist(new uint32_t[(uint64_t)nt * (RB + BB)]);
    auto count = [&](unsigned k) {
        uint32_t* rr = hist.get() + (uint64_t)k * (RB + BB);
        uint32_t* bb = rr + RB;
        memset(rr, 0, 4ull * (RB + BB));
        for (uint64_t row = T * k / nt; row < T * (k + 1) / nt; ++row) {
            const uint64_t* q = rec + 8 * row;
            const uint32_t op = (uint32_t)(q[0] >> 32) & 0xFF;
            const uint64_t iu = q[1], a = q[2], b = q[3], r = q[4], ma = q[5], mt = q[7];
            if (RB) {
                for (int j = 0; j < 4; ++j) rr[(r >> (16 * j)) & 0xFFFF] += 1;
                if (op == LD || op == SD || op == KECCAK_OP) {
                    rr[(ma >> 3) & 0xFFFF] += 1;
                    rr[8 * (ma >> 19)] += 1;
                }
                if (op == LD || op == SD) {
                    const uint64_t gap = row - mt;  // (row + 1) - mt - 1
                    rr[gap & 0xFFFF] += 1;
                    rr[gap >> 16] += 1;
                }
            }
            if (BB && op >= XOR && op <= ANDI) {
                const uint64_t second = op <= AND ? b : iu;
                const uint32_t kind = (op == XOR || op == XORI) ? 0 : (op == OR || op == ORI) ? 1 : 2;
                for (int i = 0; i < 8; ++i)
                    bb[kind * 65536 + ((((a >> (8 * i)) & 0xFF) << 8) | ((second >> (8 * i)) & 0xFF))] += 1;
            }
        }
    };
    auto merge = [&](unsigned k) {
        const uint32_t nb = RB + BB, v0 = (uint32_t)((uint64_t)nb * k / nt), v1 = (uint32_t)((uint64_t)nb * (k + 1) / nt);
        for (uint32_t v = v0; v < v1; ++v) {
            uint64_t sum = 0;
            for (unsigned j = 0; j < nt; ++j) sum += hist[(uint64_t)j * nb + v];
            if (v < RB)
                range_counts[v] += sum;
            else
                bitwise_counts[v - RB] += sum;
        }
    };
    for (auto phase : {0, 1}) {
        std::vector<std::thread> pool;
        for (unsigned k = 1; k < nt; ++k) pool.emplace_back([&, k, phase] { phase ? merge(k) : count(k); });
        phase ? merge(0) : count(0);
        for (auto& th : pool) th.join();
    }
}

// A row record is written once and read back only by other threads and the
// device upload, long after: on x86-64 it goes out with non-temporal stores,
// which skip reading the line into the cache first (the records are larger
// than the last-level cache). records_done orders those stores before any
// later read.
inline void put_record(uint64_t* q, uint64_t w0, uint64_t w1, uint64_t w2, uint64_t w3, uint64_t w4, uint64_t w5,
                       uint64_t w6, uint64_t w7) {
#if defined(__x86_64__)
    long long* p = (long long*)q;
    _mm_stream_si64(p, (long long)w0), _mm_stream_si64(p + 1, (long long)w1);
    _mm_stream_si64(p + 2, (long long)w2), _mm_stream_si64(p + 3, (long long)w3);
    _mm_stream_si64(p + 4, (long long)w4), _mm_stream_si64(p + 5, (long long)w5);
    _mm_stream_si64(p + 6, (long long)w6), _mm_stream_si64(p + 7, (long long)w7);
#else
    q[0] = w0, q[1] = w1, q[2] = w2, q[3] = w3, q[4] = w4, q[5] = w5, q[6] = w6, q[7] = w7;
#endif
}
inline void records_done() {
#if defined(__x86_64__)
    _mm_sfence();
#endif
}

// Where a run's outputs go. FixedOut: the caller's arrays, sized from an
// earlier run without outputs (sg_rv64_run / sg_rv64_run_counted). GrowOut:
// buffers that grow as the machine runs (sg_rv64_exec), so one run suffices;
// the row records live in an anonymous mapping grown with mremap, which moves
// page tables rather than copying the records.
struct FixedOut {
    uint64_t n_rows;
    uint64_t *rows, *regs, *counts, *shifts, *cells, *keccak;
    const char* fit(uint64_t t) const { return rows && t >= n_rows ? "the execution does not fit n_rows" : nullptr; }
    void snapshot(uint64_t t, const uint64_t* x) {
        if (regs && t % SG_RV64_REG_CHUNK == 0) memcpy(regs + 32 * (t / SG_RV64_REG_CHUNK), x, 256);
    }
    uint64_t* row(uint64_t t) { return rows ? rows + 8 * t : nullptr; }
    void count(uint64_t i) {
        if (counts) counts[i] += 1;
    }
    void shift(uint64_t k, uint64_t dir, uint64_t a, uint64_t amt) {
        if (shifts) shifts[3 * k] = dir, shifts[3 * k + 1] = a, shifts[3 * k + 2] = amt;
    }
    uint64_t* call(uint64_t k) { return keccak ? keccak + 52 * k : nullptr; }
    uint64_t* cell(uint64_t i) { return cells ? cells + 3 * i : nullptr; }
};

// A freed run's buffers are kept for the next run (one set, its record
// mapping up to kKeepBytes): their pages stay mapped, so a later run of a
// similar size writes without first-touch faults or vector growth (on the
// 1 MiB Keccak guest the faults cost more than writing the records).
constexpr uint64_t kKeepBytes = 8ull << 30;

struct GrowOut {
    uint64_t* rows = nullptr;
    uint64_t cap = 0;  // rows the mapping holds
    std::vector<uint64_t> regs, counts, shifts, cells, keccak, range, bitwise;

    static std::mutex& keep_mu() {
        static std::mutex m;
        return m;
    }
    static GrowOut& kept() {  // the kept buffers (never destroyed: they only ever move)
        static GrowOut* k = new GrowOut(false);
        return *k;
    }
    explicit GrowOut(bool take = true) {
        if (!take) return;
        std::lock_guard<std::mutex> g(keep_mu());
        swap_buffers(kept());
        for (auto* v : {&regs, &counts, &shifts, &cells, &keccak, &range, &bitwise}) v->clear();
    }
    ~GrowOut() {
        if (rows && cap * 64 <= kKeepBytes) {
            std::lock_guard<std::mutex> g(keep_mu());
            if (cap >= kept().cap) swap_buffers(kept());  // keep the larger set; free the other below
        }
        if (rows) munmap(rows, cap * 64);
    }
    void swap_buffers(GrowOut& o) {
        std::swap(rows, o.rows), std::swap(cap, o.cap);
        regs.swap(o.regs), counts.swap(o.counts), shifts.swap(o.shifts), cells.swap(o.cells);
        keccak.swap(o.keccak), range.swap(o.range), bitwise.swap(o.bitwise);
    }
    const char* fit(uint64_t t) {
        if (t < cap) return nullptr;
        const uint64_t ncap = cap ? 2 * cap : 1ull << 16;
        void* p = rows ? mremap(rows, cap * 64, ncap * 64, MREMAP_MAYMOVE)
                       : mmap(nullptr, ncap * 64, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (p == MAP_FAILED) return "out of host memory for the row records";
        madvise(p, ncap * 64, MADV_HUGEPAGE);  // fewer first-touch faults; advice only
        rows = (uint64_t*)p;
        cap = ncap;
        return nullptr;
    }
    void snapshot(uint64_t t, const uint64_t* x) {
        if (t % SG_RV64_REG_CHUNK == 0) regs.insert(regs.end(), x, x + 32);
    }
    uint64_t* row(uint64_t t) { return rows + 8 * t; }
    void count(uint64_t i) { counts[i] += 1; }
    void shift(uint64_t, uint64_t dir, uint64_t a, uint64_t amt) {
        shifts.push_back(dir), shifts.push_back(a), shifts.push_back(amt);
    }
    uint64_t* call(uint64_t k) {
        keccak.resize(52 * (k + 1));
        return keccak.data() + 52 * k;
    }
    uint64_t* cell(uint64_t i) {
        if (cells.size() < 3 * (i + 1)) cells.resize(3 * (i + 1));
        return cells.data() + 3 * i;
    }
};

// The machine, writing into `o`. n_rows: the table height the fill past the
// halt targets (the FixedOut's; for GrowOut 0: the power of two >= the run).
template <class O>
int run_machine(const uint32_t* words, uint32_t nwords, uint64_t max_steps, uint64_t n_rows, bool want_rows, O& o,
                uint64_t* counts, uint64_t* range_counts, uint64_t* bitwise_counts, sg_rv64_info* info) {
    std::vector<Ins> prog(nwords);
    for (uint32_t i = 0; i < nwords; ++i) SG_CHECK_ARG(decode(words[i], &prog[i]), "unsupported instruction word");
    if (counts) memset(counts, 0, nwords * sizeof(uint64_t));
    uint64_t x[32] = {0};
    uint64_t pc = 0, t = 0, nshift = 0, ncall = 0;
    uint32_t chips = 0;
    Memory mem;
    uint64_t ncells = 0;
    auto cell = [&](uint64_t addr, Cell** c) {
        if (addr % 8 || addr >> 32) return false;
        *c = mem.at(addr);  // a new cell is (0, timestamp 0)
        ncells += (*c)->stamp == 0;
        return true;
    };
    if (range_counts) memset(range_counts, 0, 65536 * 8);
    if (bitwise_counts) memset(bitwise_counts, 0, 3 * 65536 * 8);
    bool halted = false;
    while (!halted) {
        SG_CHECK_ARG(t < max_steps, "the program did not halt within max_steps");
        SG_CHECK_ARG(pc % 4 == 0 && pc / 4 < nwords, "pc outside the program");
        if (want_rows) {
            const char* why = o.fit(t);
            SG_CHECK_ARG(!why, why);
        }
        o.snapshot(t, x);
        const Ins& in = prog[pc / 4];
        const uint64_t a = x[in.rs1], b = x[in.rs2], iu = (uint64_t)in.imm, clk = t + 1;
        uint64_t r = 0, npc = pc + 4, ma = 0, mv = 0, mt = 0;
        int op = in.op;
        switch (in.op) {
            case ADD: r = a + b; break;
            case SUB: r = a - b; break;
            case XOR: r = a ^ b; break;
            case OR: r = a | b; break;
            case AND: r = a & b; break;
            case ADDI: r = a + iu; break;
            case XORI: r = a ^ iu; break;
            case ORI: r = a | iu; break;
            case ANDI: r = a & iu; break;
            case SLLI: r = a << in.imm; break;
            case SRLI: r = a >> in.imm; break;
            case LUI: r = iu; break;
            case LD:
            case SD: {
                ma = a + iu;
                Cell* c;
                SG_CHECK_ARG(cell(ma, &c), "load / store address unaligned or outside the data space");
                mv = c->value, mt = c->stamp;
                if (in.op == LD) r = mv;
                *c = Cell{in.op == LD ? mv : b, clk};
                break;
            }
            case BEQ: npc = a == b ? pc + iu : pc + 4; break;
            case BNE: npc = a != b ? pc + iu : pc + 4; break;
            case ECALL:
                if (x[17] == EXIT_CALL) {
                    halted = true;
                    npc = pc;
                } else {
                    SG_CHECK_ARG(x[17] == KECCAK_CALL, "unsupported ecall (a7 is neither 93 nor 2^64 - 2)");
                    op = KECCAK_OP;
                    ma = x[10];
                    uint64_t lanes[25];
                    Cell* cs[25];
                    for (int i = 0; i < 25; ++i) {
                        SG_CHECK_ARG(cell(ma + 8 * (uint64_t)i, &cs[i]), "keccak state unaligned or outside the data space");
                        lanes[i] = cs[i]->value;
                    }
                    if (uint64_t* k = o.call(ncall)) {
                        k[0] = clk, k[1] = ma;
                        for (int i = 0; i < 25; ++i) k[2 + i] = lanes[i], k[27 + i] = cs[i]->stamp;
                    }
                    if (range_counts)  // the KECCAK table's reads: the gaps to the cells' last accesses
                        for (int i = 0; i < 25; ++i) {
                            const uint64_t gap = clk - cs[i]->stamp - 1;
                            range_counts[gap & 0xFFFF] += 1;
                            range_counts[gap >> 16] += 1;
                        }
                    keccak_f(lanes);
                    for (int i = 0; i < 25; ++i) *cs[i] = Cell{lanes[i], clk};
                    ++ncall;
                }
                break;
        }
        if (op == SLLI || op == SRLI) {
            o.shift(nshift, op == SRLI, a, iu);
            ++nshift;
            chips |= SG_RV64_CHIP_SHIFT;
        } else if (op >= XOR && op <= ANDI) {
            chips |= SG_RV64_CHIP_BITWISE;
        } else if (op == LD || op == SD) {
            chips |= SG_RV64_CHIP_MEMORY;
        } else if (op == KECCAK_OP) {
            chips |= SG_RV64_CHIP_MEMORY | SG_RV64_CHIP_KECCAK;
        }
        if (want_rows)
            put_record(o.row(t),
                       pc | ((uint64_t)op << 32) | ((uint64_t)in.rd << 40) | ((uint64_t)in.rs1 << 48) |
                           ((uint64_t)in.rs2 << 56),
                       iu, a, b, r, ma, mv, mt);
        o.count(pc / 4);
        const bool writes = !(in.op == BEQ || in.op == BNE || in.op == ECALL || in.op == SD);
        if (in.rd && writes) x[in.rd] = r;
        pc = npc;
        ++t;
    }
    records_done();
    info->cycles = t;
    info->a0 = x[10];
    info->shifts = nshift;
    info->cells = ncells;
    info->keccak_calls = ncall;
    info->chips = chips;
    if (want_rows) {
        if (!n_rows) n_rows = std::max<uint64_t>(2, 1ull << (64 - __builtin_clzll(t - 1 | 1)));
        // the halting row repeats to fill the table, with the final registers
        if (counts) counts[pc / 4] += n_rows - t;
        if (range_counts) range_counts[0] += 4 * (n_rows - t);  // its zero result
        for (uint64_t r = (t + SG_RV64_REG_CHUNK - 1) / SG_RV64_REG_CHUNK * SG_RV64_REG_CHUNK; r < n_rows;
             r += SG_RV64_REG_CHUNK)
            o.snapshot(r, x);
        if (range_counts || bitwise_counts) count_cpu_lookups(o.row(0), t, range_counts, bitwise_counts);
    }
    uint64_t i = 0;
    mem.each_touched([&](uint64_t addr, const Cell& c) {
        if (uint64_t* q = o.cell(i)) q[0] = addr, q[1] = c.value, q[2] = c.stamp;
        ++i;
    });
    return SG_OK;
}

}  // namespace

using namespace sg;

// One run's outputs, owned by the library (sg_rv64_exec).
struct sg_rv64_trace {
    GrowOut out;
    sg_rv64_info info;
};

extern "C" int sg_rv64_run(const uint32_t* words, uint32_t nwords, uint64_t max_steps, uint64_t n_rows,
                           uint64_t* rows_out, uint64_t* regs_out, uint64_t* counts_out, uint64_t* shifts_out,
                           uint64_t* cells_out, uint64_t* keccak_out, sg_rv64_info* info) {
    return sg_rv64_run_counted(words, nwords, max_steps, n_rows, rows_out, regs_out, counts_out, shifts_out, cells_out,
                               keccak_out, nullptr, nullptr, info);
}

extern "C" int sg_rv64_run_counted(const uint32_t* words, uint32_t nwords, uint64_t max_steps, uint64_t n_rows,
                                   uint64_t* rows_out, uint64_t* regs_out, uint64_t* counts_out, uint64_t* shifts_out,
                                   uint64_t* cells_out, uint64_t* keccak_out, uint64_t* range_counts,
                                   uint64_t* bitwise_counts, sg_rv64_info* info) {
    SG_CHECK_ARG(words && nwords && info, "null argument");
    SG_CHECK_ARG(!rows_out || (n_rows >= 2 && (n_rows & (n_rows - 1)) == 0), "n_rows must be a power of two >= 2");
    SG_CHECK_ARG(!range_counts || rows_out, "lookup counts need the n_rows table");
    SG_CHECK_ARG(!bitwise_counts || rows_out, "lookup counts need the n_rows table");
    FixedOut o{n_rows, rows_out, regs_out, counts_out, shifts_out, cells_out, keccak_out};
    return run_machine(words, nwords, max_steps, n_rows, rows_out != nullptr, o, counts_out, range_counts,
                       bitwise_counts, info);
}

extern "C" int sg_rv64_exec(const uint32_t* words, uint32_t nwords, uint64_t max_steps, sg_rv64_trace** out,
                            sg_rv64_info* info) {
    SG_CHECK_ARG(words && nwords && out && info, "null argument");
    *out = nullptr;
    sg_rv64_trace* tr = new (std::nothrow) sg_rv64_trace();
    SG_CHECK_ARG(tr, "out of host memory");
    GrowOut& o = tr->out;
    o.counts.assign(nwords, 0);
    o.range.assign(65536, 0);
    o.bitwise.assign(3 * 65536, 0);
    const int rc = run_machine(words, nwords, max_steps, 0, true, o, o.counts.data(), o.range.data(),
                               o.bitwise.data(), info);
    if (rc != SG_OK) {
        delete tr;
        return rc;
    }
    tr->info = *info;
    *out = tr;
    return SG_OK;
}

extern "C" int sg_rv64_trace_part(const sg_rv64_trace* tr, uint32_t part, const uint64_t** data, uint64_t* words) {
    SG_CHECK_ARG(tr && data && words, "null argument");
    const GrowOut& o = tr->out;
    switch (part) {
        case SG_RV64_PART_ROWS: *data = o.rows, *words = 8 * tr->info.cycles; break;
        case SG_RV64_PART_REGS: *data = o.regs.data(), *words = o.regs.size(); break;
        case SG_RV64_PART_COUNTS: *data = o.counts.data(), *words = o.counts.size(); break;
        case SG_RV64_PART_SHIFTS: *data = o.shifts.data(), *words = o.shifts.size(); break;
        case SG_RV64_PART_CELLS: *data = o.cells.data(), *words = o.cells.size(); break;
        case SG_RV64_PART_KECCAK: *data = o.keccak.data(), *words = o.keccak.size(); break;
        case SG_RV64_PART_RANGE_COUNTS: *data = o.range.data(), *words = o.range.size(); break;
        case SG_RV64_PART_BITWISE_COUNTS: *data = o.bitwise.data(), *words = o.bitwise.size(); break;
        default: SG_CHECK_ARG(false, "unknown trace part");
    }
    return SG_OK;
}

extern "C" void sg_rv64_trace_free(sg_rv64_trace* tr) { delete tr; }

// ---------------------------------------------------------------------------
// Chip tables expanded on the device from the run's compact events, so the
// host never writes or uploads them: the KECCAK table (24 rows x 2605 columns
// per ecall from 52 words of event) and the SHIFT table (148 columns per
// shift from 3 words). Layouts: rv64_air.py's KeccakAir and ShiftAir.
namespace {

constexpr int KW = 2605;  // KECCAK table columns
constexpr int K_A = 24, K_C = 124, K_CP = 444, K_AP = 764, K_OUT = 2364, K_B00 = 2464, K_BASE = 2528, K_CLK = 2529,
              K_TOLD = 2530, K_TD = 2555;
constexpr int K_SLOTS = 86;  // per round: A[25], C[5], C'[5], A'[25], OUT[25], chi lane 0 before iota

// One CTA per ecall: thread 0 runs the 24 rounds into shared memory, then the
// CTA writes the ecall's 24 rows, consecutive threads on consecutive columns.
__global__ void k_keccak_rows(const uint64_t* __restrict__ calls, uint64_t count, KeccakConsts kc,
                              uint64_t* __restrict__ out) {
    __shared__ uint64_t s[24][K_SLOTS];
    for (uint64_t p = blockIdx.x; p < count; p += gridDim.x) {
        const uint64_t* ev = calls + 52 * p;
        if (threadIdx.x == 0) {
            uint64_t a[25];
            for (int i = 0; i < 25; ++i) a[i] = ev[2 + i];
            for (int r = 0; r < 24; ++r) {
                uint64_t* o = s[r];
                uint64_t c[5], d[5], b[25];
                for (int x = 0; x < 5; ++x) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
                for (int x = 0; x < 5; ++x) {
                    const uint64_t n1 = c[(x + 1) % 5];
                    d[x] = c[(x + 4) % 5] ^ ((n1 << 1) | (n1 >> 63));
                }
                for (int i = 0; i < 25; ++i) {
                    o[i] = a[i];
                    o[55 + i] = 0;
                }
                for (int x = 0; x < 5; ++x) o[25 + x] = c[x], o[30 + x] = c[x] ^ d[x];
                for (int x = 0; x < 5; ++x)
                    for (int y = 0; y < 5; ++y) {
                        const uint64_t v = a[x + 5 * y] ^ d[x];
                        o[35 + x + 5 * y] = v;
                        const int rr = kc.rot[x + 5 * y];
                        b[y + 5 * ((2 * x + 3 * y) % 5)] = rr ? (v << rr) | (v >> (64 - rr)) : v;
                    }
                for (int x = 0; x < 5; ++x)
                    for (int y = 0; y < 5; ++y)
                        a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
                o[85] = a[0];
                a[0] ^= kc.rc[r];
                for (int i = 0; i < 25; ++i) o[60 + i] = a[i];
            }
        }
        __syncthreads();
        const uint64_t clk = ev[0], base = ev[1];
        uint64_t* rows = out + 24 * p * (uint64_t)KW;
        for (uint32_t idx = threadIdx.x; idx < 24u * KW; idx += blockDim.x) {
            const uint32_t r = idx / KW, c = idx % KW;
            const uint64_t* o = s[r];
            uint64_t v;
            if (c < K_A) v = c == r;
            else if (c < K_C) v = (o[(c - K_A) / 4] >> (16 * ((c - K_A) % 4))) & 0xFFFF;
            else if (c < K_CP) v = (o[25 + (c - K_C) / 64] >> ((c - K_C) % 64)) & 1;
            else if (c < K_AP) v = (o[30 + (c - K_CP) / 64] >> ((c - K_CP) % 64)) & 1;
            else if (c < K_OUT) v = (o[35 + (c - K_AP) / 64] >> ((c - K_AP) % 64)) & 1;
            else if (c < K_B00) v = (o[60 + (c - K_OUT) / 4] >> (16 * ((c - K_OUT) % 4))) & 0xFFFF;
            else if (c < K_BASE) v = (o[85] >> (c - K_B00)) & 1;
            else if (c == K_BASE) v = base;
            else if (c == K_CLK) v = clk;
            else if (c < K_TD) v = r == 0 ? ev[27 + (c - K_TOLD)] : 0;
            else {
                const uint32_t j = c - K_TD;
                const uint64_t gap = clk - ev[27 + j / 2] - 1;
                v = r == 0 ? ((j & 1) ? gap >> 16 : gap & 0xFFFF) : 0;
            }
            rows[idx] = v;
        }
        __syncthreads();
    }
}

constexpr int SW = 148;  // SHIFT table columns: DIR, bits of a (64), S (8), Q (8), bits of a >>/<< s (64), R_LO, R_HI, M

__global__ void k_shift_rows(const uint64_t* __restrict__ ev, uint64_t count, uint64_t n_rows,
                             uint64_t* __restrict__ out) {
    const uint64_t total = n_rows * SW;
    for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = idx / SW;
        const uint32_t c = (uint32_t)(idx % SW);
        uint64_t v;
        if (row >= count) {
            v = (c == 65 || c == 73);  // padding: a = 0, k = 0
        } else {
            const uint64_t dir = ev[3 * row], a = ev[3 * row + 1], k = ev[3 * row + 2];
            const uint64_t sb = k & 7, q = k >> 3;
            const uint64_t t = dir ? a >> sb : a << sb, res = dir ? a >> k : a << k;
            if (c == 0) v = dir;
            else if (c < 65) v = (a >> (c - 1)) & 1;
            else if (c < 73) v = (c - 65) == sb;
            else if (c < 81) v = (c - 73) == q;
            else if (c < 145) v = (t >> (c - 81)) & 1;
            else if (c == 145) v = res & M32;
            else if (c == 146) v = res >> 32;
            else v = 1;
        }
        out[idx] = v;
    }
}

// (a - b) mod p of two values below 2^32
__device__ __forceinline__ uint64_t sub_small(uint64_t a, uint64_t b) { return a >= b ? a - b : GL_P - (b - a); }

// One cell of the CPU table outside the register file, from the row's record.
__device__ uint64_t cpu_cell(uint32_t c, uint64_t row, uint64_t n_rows, uint32_t op, uint64_t pc, uint32_t rd,
                             uint32_t rs1, uint32_t rs2, uint64_t imm, uint64_t a, uint64_t b, uint64_t r, uint64_t ma,
                             uint64_t mv, uint64_t mt) {
    if (c == PC) return pc;
    if (c == STEP) return row + 1 != n_rows;
    if (c == CLK) return row + 1;
    if (c < RD0) return c - SEL0 + 1 == op;
    if (c < RS10) return c - RD0 == rd;
    if (c < RS20) return c - RS10 == rs1;
    if (c < IMM_LO) return c - RS20 == rs2;
    switch (c) {
        case IMM_LO: return imm & M32;
        case IMM_HI: return imm >> 32;
        case IMM_F: return (int64_t)imm < 0 ? GL_P - (uint64_t)(-(int64_t)imm) : imm;
        case A_LO: return a & M32;
        case A_HI: return a >> 32;
        case B_LO: return b & M32;
        case B_HI: return b >> 32;
        case R_LO: return r & M32;
        case R_HI: return r >> 32;
        case R16: case R16 + 1: case R16 + 2: case R16 + 3: return (r >> (16 * (c - R16))) & 0xFFFF;
        case C0: case C1: {
            if (op == ADD || op == ADDI || op == LD || op == SD) {
                const uint64_t o = op == ADD ? b : imm;
                const uint64_t c0 = ((a & M32) + (o & M32)) >> 32;
                return c == C0 ? c0 : ((a >> 32) + (o >> 32) + c0) >> 32;
            }
            if (op == SUB) {
                const uint64_t b0 = (a & M32) < (b & M32);
                return c == C0 ? b0 : (uint64_t)((a >> 32) < (b >> 32) + b0);
            }
            return 0;
        }
        default: break;
    }
    if (c <= BR) {  // INV_LO .. BR: the branch witnesses
        if (op != BEQ && op != BNE) return 0;
        const uint64_t dl = sub_small(a & M32, b & M32), dh = sub_small(a >> 32, b >> 32);
        const uint64_t ne = (dl != 0) | (dh != 0);
        switch (c) {
            case INV_LO: return dl ? gl::canon(gl::inv(dl)) : 0;
            case INV_HI: return dh ? gl::canon(gl::inv(dh)) : 0;
            case E_LO: return dl != 0;
            case E_HI: return dh != 0;
            case NE: return ne;
            default: return op == BNE ? ne : 1 - ne;
        }
    }
    if (c < MA) {  // bytes of a, of the second operand and of the result (bitwise ops)
        if (op < XOR || op > ANDI) return 0;
        const uint32_t i = (c - AB0) % 8;
        const uint64_t v = c < BB0 ? a : c < RB0 ? (op <= AND ? b : imm) : r;
        return (v >> (8 * i)) & 0xFF;
    }
    const bool mem = op == LD || op == SD;
    switch (c) {
        case MA: return mem || op == KECCAK_OP ? ma : 0;
        case MW0: return mem || op == KECCAK_OP ? (ma >> 3) & 0xFFFF : 0;
        case MW1: return mem || op == KECCAK_OP ? ma >> 19 : 0;
        case MV_LO: return mem ? mv & M32 : 0;
        case MV_HI: return mem ? mv >> 32 : 0;
        case MT: return mem ? mt : 0;
        case MD0: return mem ? (row - mt) & 0xFFFF : 0;  // (row + 1) - mt - 1
        case MD1: return mem ? (row - mt) >> 16 : 0;
        case NV_LO: return op == LD ? mv & M32 : op == SD ? b & M32 : 0;
        default: return op == LD ? mv >> 32 : op == SD ? b >> 32 : 0;  // NV_HI
    }
}

// One warp per chunk of SG_RV64_REG_CHUNK rows: lane k holds register x_k
// (from the chunk's snapshot) and the warp walks the chunk's rows in order,
// writing each row's register columns by shuffles and its other columns
// lane-strided, then applying the row's register write. Rows past the
// execution repeat the halting row's record with their own timestamps.
__global__ void k_cpu_rows(const uint64_t* __restrict__ recs, uint64_t T, const uint64_t* __restrict__ regs,
                           uint64_t n_rows, uint32_t width, uint64_t* __restrict__ out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t nchunks = (n_rows + SG_RV64_REG_CHUNK - 1) / SG_RV64_REG_CHUNK;
    const uint32_t k1 = lane / 2 + 1, k2 = lane < 30 ? (lane + 32) / 2 + 1 : 31;
    for (uint64_t ch = warp; ch < nchunks; ch += nwarps) {
        uint64_t xr = regs[32 * ch + lane];
        const uint64_t r0 = ch * SG_RV64_REG_CHUNK;
        const uint64_t r1 = r0 + SG_RV64_REG_CHUNK < n_rows ? r0 + SG_RV64_REG_CHUNK : n_rows;
        for (uint64_t row = r0; row < r1; ++row) {
            const uint64_t* q = recs + 8 * (row < T ? row : T - 1);
            const uint64_t w0 = q[0], imm = q[1], a = q[2], b = q[3], r = q[4], ma = q[5], mv = q[6], mt = q[7];
            const uint32_t op = (uint32_t)(w0 >> 32) & 0xFF, rd = (uint32_t)(w0 >> 40) & 0xFF,
                           rs1 = (uint32_t)(w0 >> 48) & 0xFF, rs2 = (uint32_t)(w0 >> 56);
            uint64_t* o = out + row * width;
            const uint64_t v1 = __shfl_sync(0xFFFFFFFFu, xr, k1), v2 = __shfl_sync(0xFFFFFFFFu, xr, k2);
            o[X0 + lane] = (lane & 1) ? v1 >> 32 : v1 & M32;
            if (lane < 30) o[X0 + 32 + lane] = (lane & 1) ? v2 >> 32 : v2 & M32;
            for (uint32_t c = lane; c < width; c += 32) {
                if (c >= (uint32_t)X0 && c < (uint32_t)X0 + 62) continue;
                o[c] = cpu_cell(c, row, n_rows, op, w0 & M32, rd, rs1, rs2, imm, a, b, r, ma, mv, mt);
            }
            const bool writes = row < T && !(op == BEQ || op == BNE || op == ECALL || op == SD || op == KECCAK_OP);
            if (writes && rd != 0 && lane == rd) xr = r;
        }
    }
}

// MEMORY table rows (ADDR, V_LO, V_HI, T, ACT, NW, D0, D1; rv64_air.py's
// MemoryAir) from `count` touched cells (address, final value, final
// timestamp) in ascending address order; rows past the cells continue the
// addresses in steps of 8, and every row but the last steps to the next.
constexpr int MW = 8;
static_assert(MW == SG_RV64_MEMORY_WIDTH, "MEMORY table width");
__global__ void k_memory_rows(const uint64_t* __restrict__ cells, uint64_t count, uint64_t n_rows,
                              uint64_t* __restrict__ out) {
    const uint64_t last = cells[3 * (count - 1)];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_rows;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const bool act = i < count;
        const uint64_t a = act ? cells[3 * i] : last + 8 * (i - count + 1);
        const uint64_t v = act ? cells[3 * i + 1] : 0, t = act ? cells[3 * i + 2] : 0;
        uint64_t d = 0;
        if (i + 1 < n_rows) d = ((i + 1 < count ? cells[3 * (i + 1)] : last + 8 * (i + 2 - count)) - a - 8) >> 3;
        uint64_t* o = out + MW * i;
        o[0] = a, o[1] = v & M32, o[2] = v >> 32, o[3] = t;
        o[4] = act, o[5] = i + 1 < n_rows, o[6] = d & 0xFFFF, o[7] = d >> 16;
    }
}

int upload_events(Ctx* ctx, cudaStream_t st, const uint64_t* host, uint64_t words, uint64_t** d,
                  const std::function<bool(uint64_t lo, uint64_t hi)>& check = nullptr) {
    SG_TRY(dev_alloc(ctx, st, 8 * words, (void**)d));
    const int rc = upload_host(ctx, st, host, 8 * words, *d, check);
    if (rc != SG_OK) {
        dev_free(ctx, st, *d, 8 * words);
        set_error(std::string("rv64: event upload failed: ") + last_error());
        return rc;
    }
    return SG_OK;
}

}  // namespace

extern "C" int sg_rv64_cpu_table(sg_ctx* c, void* stream, const uint64_t* rows, uint64_t count, const uint64_t* regs,
                                 uint64_t n_rows, uint32_t width, uint64_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && d_out && rows && regs, "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(count >= 1 && count <= n_rows, "the execution does not fit n_rows");
    SG_CHECK_ARG(width == SG_RV64_CPU_CORE_WIDTH || width == SG_RV64_CPU_WIDTH, "width is the core or the full width");
    // 0: good; 1: a bad record; 2: a chip instruction in a core-width table
    // the records are checked by the threads that stage them for the upload
    // (each record whose first byte falls in the range it copies): 1 a bad
    // record, 2 a chip instruction in a core-width table
    std::atomic<int> bad{0};
    auto check = [&](uint64_t lo, uint64_t hi) {
        int b = 0;
        for (uint64_t i = (lo + 63) / 64; i < (hi + 63) / 64 && !b; ++i) {
            const uint64_t w0 = rows[8 * i];
            const uint32_t op = (uint32_t)(w0 >> 32) & 0xFF;
            if (!(op >= 1 && op <= KECCAK_OP && ((w0 >> 40) & 0xFF) < 32 && ((w0 >> 48) & 0xFF) < 32 &&
                  (w0 >> 56) < 32))
                b = 1;
            else if (!(width == SG_RV64_CPU_WIDTH || op < XOR || op == SLLI || op == SRLI))
                b = 2;
        }
        if (b) {
            int z = 0;
            bad.compare_exchange_strong(z, b);
        }
        return b == 0;
    };
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t nchunks = (n_rows + SG_RV64_REG_CHUNK - 1) / SG_RV64_REG_CHUNK;
    uint64_t *d_rows = nullptr, *d_regs = nullptr;
    int rc0 = upload_events(ctx, st, rows, 8 * count, &d_rows, check);
    if (rc0 != SG_OK) {
        SG_CHECK_ARG(bad.load() != 1, "bad row record");
        SG_CHECK_ARG(bad.load() != 2, "a chip instruction in a table without the chips' columns");
        return rc0;
    }
    int rc = upload_events(ctx, st, regs, 32 * nchunks, &d_regs);
    if (rc == SG_OK) {
        const uint64_t warps = nchunks < 148ull * 64 ? nchunks : 148ull * 64;
        k_cpu_rows<<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(d_rows, count, d_regs, n_rows, width, d_out);
        rc = check_launch(ctx, "k_cpu_rows");
        dev_free(ctx, st, d_regs, 8 * 32 * nchunks);
    }
    dev_free(ctx, st, d_rows, 8 * 8 * count);
    return rc;
}

extern "C" int sg_rv64_keccak_table(sg_ctx* c, void* stream, const uint64_t* calls, uint64_t count, uint64_t n_rows,
                                    uint64_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && d_out && (calls || !count), "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(count <= n_rows / 24, "the ecalls do not fit n_rows");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t used = 24 * count;
    if (used < n_rows && cudaMemsetAsync(d_out + used * KW, 0, (n_rows - used) * KW * 8, st) != cudaSuccess) {
        set_error("rv64: padding fill failed");
        return SG_ERR_CUDA;
    }
    if (!count) return SG_OK;
    const KeccakConsts kc = keccak_consts();
    uint64_t* d_ev = nullptr;
    SG_TRY(upload_events(ctx, st, calls, 52 * count, &d_ev));
    const unsigned grid = (unsigned)std::min<uint64_t>(count, 148ull * 16);
    k_keccak_rows<<<grid, 256, 0, st>>>(d_ev, count, kc, d_out);
    const int rc = check_launch(ctx, "k_keccak_rows");
    dev_free(ctx, st, d_ev, 8 * 52 * count);
    return rc;
}

extern "C" int sg_rv64_shift_table(sg_ctx* c, void* stream, const uint64_t* shifts, uint64_t count, uint64_t n_rows,
                                   uint64_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && d_out && (shifts || !count), "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(count <= n_rows, "the shifts do not fit n_rows");
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t* d_ev = nullptr;
    // the events are checked by the threads that stage them (each whose first byte falls in the range)
    std::atomic<bool> bad{false};
    auto check = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = (lo + 23) / 24; i < (hi + 23) / 24; ++i)
            if (shifts[3 * i] > 1 || shifts[3 * i + 2] >= 64) return !(bad = true);
        return true;
    };
    if (count) {
        const int rc0 = upload_events(ctx, st, shifts, 3 * count, &d_ev, check);
        SG_CHECK_ARG(!bad.load(), "bad shift event");
        SG_TRY(rc0);
    }
    const uint64_t total = n_rows * SW;
    const unsigned grid = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
    k_shift_rows<<<grid, 256, 0, st>>>(d_ev, count, n_rows, d_out);
    const int rc = check_launch(ctx, "k_shift_rows");
    if (d_ev) dev_free(ctx, st, d_ev, 8 * 3 * count);
    return rc;
}

extern "C" int sg_rv64_memory_table(sg_ctx* c, void* stream, const uint64_t* cells, uint64_t count, uint64_t n_rows,
                                    uint64_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && d_out && cells, "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(count >= 1 && count <= n_rows && n_rows <= (1ull << 32), "the cells do not fit n_rows");
    std::atomic<bool> bad{false};
    host_parallel(count, 1 << 16, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            const uint64_t a = cells[3 * i];
            if (a % 8 || a >> 32 || (i && a <= cells[3 * (i - 1)])) {
                bad = true;
                return;
            }
        }
    });
    SG_CHECK_ARG(!bad.load(), "cell addresses must be ascending multiples of 8 below 2^32");
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t* d_ev = nullptr;
    SG_TRY(upload_events(ctx, st, cells, 3 * count, &d_ev));
    const unsigned grid = (unsigned)std::min<uint64_t>((n_rows + 255) / 256, 148ull * 16);
    k_memory_rows<<<grid, 256, 0, st>>>(d_ev, count, n_rows, d_out);
    const int rc = check_launch(ctx, "k_memory_rows");
    dev_free(ctx, st, d_ev, 8 * 3 * count);
    return rc;
}
