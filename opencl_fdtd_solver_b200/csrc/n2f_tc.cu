// Near-to-far contraction on the tensor cores (tcgen05, TMEM accumulators).
//
// The far-field integrals of the reference (farfield_accumulate_nl,
// dft_farfield.cl:372-556) are, per direction r̂_o, frequency f and face,
//   NL_face(o, c) = Σ_{p,q} e^{jk r̂_o·r'_{pq}} cur[p][q][c],
// with k = 2πf/c0, c over the face's four tangential currents (J_b, J_c, M_b,
// M_c; b, c the in-face axes) and r'_{pq} = x_n n̂ + (o_p + p·h) b̂ + (o_q + q·h) ĉ.
// The phase separates: e^{jk r̂·r'} = C(o)·u_p(o)·v_q(o) with
//   u_p = e^{j2π γ_p p}, v_q = e^{j2π γ_q q}, γ = f·h·r̂/c0 (turns per sample),
//   C   = e^{j2π f (r̂_n x_n + r̂_b o_p + r̂_c o_q)/c0}.
// So T[o][q][c] = Σ_p u_p(o)·cur[p][q][c] is a complex GEMM (M = directions,
// K = p, N = (q, c)), and NL_face(o, c) = C(o)·Σ_q v_q(o)·T[o][q][c] is a
// row-wise reduction of its output.
//
// Kernel k_n2f_tc: one CTA per (128-direction tile, face, frequency), 6 + 4·NGRP warps.
//   * warp 0: B producer.  B (currents, N × K) is pre-packed by k_n2f_pack in
//     the K-major core-matrix layout, one contiguous 32 KB block per
//     (n tile, K step) in both modes, and moved with one cp.async.bulk per
//     stage (no tensor map, no multicast).
//   * warp 1: one thread issues tcgen05.mma (kind::f16 BF16: hi·hi + hi·lo +
//     lo·hi, or kind::tf32), MPS K groups per stage (2 BF16, 4 TF32), into a 128 × 256 FP32
//     accumulator in TMEM, double-buffered across n tiles (512 columns).
//   * warps 2-5 and 10 onwards: A (phases, 128 × K), generated in shared memory
//     per K step, one direction per thread, NGRP groups on interleaved stages: a
//     float64 rotation times PS (16) precomputed float phases, split into
//     bf16 hi + lo (or rounded to tf32), written in the K-major core-matrix
//     layout.
//   * warps 6-9: epilogue.  Each thread owns one TMEM lane (one direction),
//     reads it with tcgen05.ld and folds Σ_q v_q·T into four complex sums while
//     the next n tile's MMAs run.
// Complex arithmetic in real GEMM form: K interleaves (Re, Im) of u_p and N
// interleaves (Re, Im) of T, with B = [[Br, Bi], [−Bi, Br]] per (p, (q, c)).
//
// Every mbarrier wait is bounded in wall time (Params::wait_ns, 0.2 s by
// default; fdtd_set_wait_budget lowers it); on timeout the kernel raises bit 1
// of the device error flag, stops issuing, drains its own copies and MMAs (with
// the default bound), frees TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "launch_count.cuh"
#include "n2f.cuh"

namespace fdtd {
namespace n2f {

__device__ int g_n2f_error;

constexpr int NGRP = 2;  // phase-generator groups of four warps, on stages g % NGRP
constexpr int NTHREADS = (6 + 4 * NGRP) * 32;  // B loader, MMA issuer, epilogue, phase groups
constexpr int MAX_STAGE = 16;
constexpr int ATM_NST = 6;          // stages when A is in tensor memory (6 x 32 KB of B)
constexpr uint32_t ATM_ACOL = 256;  // first TMEM column of the A ring (32 per stage)
constexpr double C0 = 299792458.0;

template <int MODE>
struct Cfg;
// A stage holds KR real K values: NCH 16-byte K chunks per operand row, MPS
// MMAs of two chunks each (K = 16 BF16 or 8 TF32 per MMA).  Wider stages
// amortise the per-stage barrier round trips over more MMAs.
template <>
struct Cfg<FDTD_N2F_BF16X3> {
    static constexpr int KR = 32;                 // real K per stage
    static constexpr int PS = KR / 2;             // complex samples p per stage
    static constexpr int NCH = KR / 8;            // 16-byte chunks per row
    static constexpr int MPS = NCH / 2;           // MMA K groups per stage
    static constexpr int A_BYTES = BM * KR * 2;   // one of hi / lo
    static constexpr int B_BYTES = BN * KR * 2;   // one of hi / lo
    static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int B_COPY = 2 * B_BYTES;
    static constexpr int NST = (192 * 1024) / STAGE;  // 192 KB of stages: one CTA per SM
    static constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};
template <>
struct Cfg<FDTD_N2F_TF32> {
    static constexpr int KR = 32;
    static constexpr int PS = KR / 2;
    static constexpr int NCH = KR / 4;
    static constexpr int MPS = NCH / 2;
    static constexpr int A_BYTES = BM * KR * 4;
    static constexpr int B_BYTES = BN * KR * 4;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int B_COPY = B_BYTES;
    static constexpr int NST = (192 * 1024) / STAGE;
    static constexpr uint32_t IDESC =
        (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};
static_assert(ATM_NST <= MAX_STAGE && ATM_ACOL + 32 * ATM_NST <= 512 && ATM_ACOL >= BN,
              "the tensor-memory A ring must fit beside one accumulator in 512 columns");
static_assert(Cfg<FDTD_N2F_BF16X3>::NST <= MAX_STAGE && Cfg<FDTD_N2F_TF32>::NST <= MAX_STAGE,
              "stage ring larger than the barrier arrays");

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Non-blocking probe of a phase (no suspension), used by a zero wait budget.
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes,
                                          uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
template <int MODE>
__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    const uint32_t z = 0;
    if (MODE == FDTD_N2F_BF16X3) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d),
            "l"(a), "l"(b), "r"(Cfg<MODE>::IDESC), "r"(acc), "r"(z)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d),
            "l"(a), "l"(b), "r"(Cfg<MODE>::IDESC), "r"(acc), "r"(z)
            : "memory");
    }
}
// The same MMA with A (M x K, one row per TMEM lane, K packed along columns)
// read from tensor memory instead of shared memory.
template <int MODE>
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t acc) {
    if (MODE == FDTD_N2F_BF16X3) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
            "r"(a_tmem), "l"(b), "r"(Cfg<MODE>::IDESC), "r"(acc)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
            "r"(a_tmem), "l"(b), "r"(Cfg<MODE>::IDESC), "r"(acc)
            : "memory");
    }
}
// Each thread of the warp writes 16 consecutive 32-bit columns of its own lane.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
        "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_st_wait() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     bar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// K-major, no-swizzle shared-memory matrix descriptor: core matrices of 8 rows
// x 16 bytes, SBO between 8-row groups, LBO between the two 16-byte K chunks.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for tcgen05
    return d;
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// e^{j2π t} for t = g·n, reduced to [-1/2, 1/2] turns in float64 first.
__device__ __forceinline__ float2 phase_turns(double g, double n) {
    double t = g * n;
    t = t - rint(t);
    float s, c;
    sincospif(2.0f * (float)t, &s, &c);
    return make_float2(c, s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// e^{j2π t} for t = g·n in float64 (reduction in turns, then sincospi).
__device__ __forceinline__ double2 zphase_turns(double g, double n) {
    double t = g * n;
    t = t - rint(t);
    double s, c;
    sincospi(2.0 * t, &s, &c);
    return make_double2(c, s);
}

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait shared by all roles: gives up after `budget_ns` of wall time
// (the launch's Params::wait_ns, 0.2 s unless a caller lowered it), when another
// role of this CTA aborted, or when another CTA raised the error flag.  Returns
// false in all three cases (and raises the flags on a timeout).  A zero budget
// gives up at once unless the phase has already completed (non-blocking probe).
constexpr uint64_t WAIT_NS = 200000000ull;  // 0.2 s; a normal wait is microseconds
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                         uint64_t budget_ns) {
    if (budget_ns == 0) {
        if (mbar_test_wait(bar, parity)) return true;
        *abort_flag = 1;
        atomicOr(&g_n2f_error, 1);
        return false;
    }
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    uint32_t it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if ((++it & 255u) == 0) {
            if (*abort_flag || *(volatile int *)&g_n2f_error) {
                *abort_flag = 1;
                return false;
            }
            if (gtimer() - t0 > budget_ns) {
                *abort_flag = 1;
                atomicOr(&g_n2f_error, 1);
                return false;
            }
        }
    }
    return true;
}

// Drain wait: bounded by time only (used before the CTA exits).
__device__ __forceinline__ void drain_bar(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = gtimer();
    while (!mbar_try_wait(bar, parity) && gtimer() - t0 < WAIT_NS) {
    }
}

struct Smem {
    uint64_t full_b[MAX_STAGE], full_a[MAX_STAGE], empty[MAX_STAGE];
    uint64_t acc_full[2], acc_empty[2];
    uint32_t tmem;
    int abort_flag;
};

// ATM: the A operand (phases) lives in tensor memory: the generators write it
// with tcgen05.st, one row (direction) per TMEM lane, and the MMAs read it from
// there, so shared memory carries only B (its copies and the MMAs' B reads).
// TMEM then holds one 128 x 256 accumulator (columns 0-255) and the A ring
// (columns 256-511, 32 per stage); without ATM the accumulator is
// double-buffered over the 512 columns and A is in the shared-memory stages.
template <int MODE, bool ATM>
__global__ void __launch_bounds__(NTHREADS, 1) k_n2f_tc(Params P) {
    using C = Cfg<MODE>;
    constexpr int NSTAGE = ATM ? ATM_NST : C::NST;
    constexpr int SSTAGE = ATM ? C::B_COPY : C::STAGE;  // shared-memory bytes per stage
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *stages = smem_raw;
    Smem *sm = reinterpret_cast<Smem *>(smem_raw + NSTAGE * SSTAGE);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = blockIdx.x, fi = blockIdx.y, fr = blockIdx.z;
    const Face &F = P.face[fi];
    const int KS = F.ks, NT = F.nt;
    const double freq = P.freqs[fr];
    volatile int *abort_flag = &sm->abort_flag;

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) {
            mbar_init(smem_u32(&sm->full_b[s]), 1);
            mbar_init(smem_u32(&sm->full_a[s]), BM);
            mbar_init(smem_u32(&sm->empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&sm->acc_full[b]), 1);
            mbar_init(smem_u32(&sm->acc_empty[b]), 128);
        }
        sm->abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(&sm->tmem), 2 * BN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm->tmem;
    const int total = NT * KS;

    if (warp == 0) {
        // ---- B producer: one bulk copy per stage
        if (lane == 0) {
            const unsigned char *src = P.btiles + F.b_off + (int64_t)fr * F.b_freq_stride;
            int issued = 0;
            for (int g = 0; g < total; ++g) {
                const int s = g % NSTAGE;
                if (g >= NSTAGE &&
                    !wait_bar(smem_u32(&sm->empty[s]), ((g / NSTAGE) - 1) & 1, abort_flag, P.wait_ns))
                    break;
                const uint32_t bar = smem_u32(&sm->full_b[s]);
                mbar_arrive_tx(bar, C::B_COPY);
                const int boff = ATM ? 0 : (MODE == FDTD_N2F_BF16X3 ? 2 : 1) * C::A_BYTES;
                bulk_load(smem_u32(stages + s * SSTAGE + boff), src + (int64_t)g * C::B_COPY,
                          C::B_COPY, bar);
                issued = g + 1;
            }
            // every issued copy has landed before the CTA may exit
            for (int g = (issued > NSTAGE ? issued - NSTAGE : 0); g < issued; ++g)
                drain_bar(smem_u32(&sm->full_b[g % NSTAGE]), (g / NSTAGE) & 1);
        }
    } else if (warp == 1) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint32_t sbase = smem_u32(stages);
            int last = -1;  // last stage whose commit was issued
            bool ok = true;
            for (int nt = 0; nt < NT && ok; ++nt) {
                // ATM: one accumulator, free once the epilogue read tile nt-1;
                // else two, buffer b free once the epilogue read tile nt-2
                const int b = ATM ? 0 : (nt & 1);
                const bool need = ATM ? nt >= 1 : nt >= 2;
                const uint32_t epar = ATM ? ((nt - 1) & 1) : (((nt >> 1) + 1) & 1);
                if (need && !wait_bar(smem_u32(&sm->acc_empty[b]), epar, abort_flag, P.wait_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * BN);
                for (int ks = 0; ks < KS; ++ks) {
                    const int g = nt * KS + ks, s = g % NSTAGE;
                    const uint32_t par = (g / NSTAGE) & 1;
                    if (!wait_bar(smem_u32(&sm->full_b[s]), par, abort_flag, P.wait_ns) ||
                        !wait_bar(smem_u32(&sm->full_a[s]), par, abort_flag, P.wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = sbase + s * SSTAGE;
#pragma unroll
                    for (int m = 0; m < C::MPS; ++m) {
                        // MMA m reads K chunks 2m and 2m+1 of the stage
                        const uint32_t ao = m * 2 * (BM / 8) * 128, bo = m * 2 * (BN / 8) * 128;
                        const uint32_t acc0 = (ks > 0 || m > 0) ? 1u : 0u;
                        if (ATM) {
                            // A of MMA m: 8 TMEM columns (16 BF16 or 8 TF32 of K) per row
                            const uint32_t a = tmem + ATM_ACOL + (uint32_t)(s * 32 + m * 8);
                            if (MODE == FDTD_N2F_BF16X3) {
                                const uint64_t bhi = make_desc(st + bo, BN * 16, 128);
                                const uint64_t blo = make_desc(st + C::B_BYTES + bo, BN * 16, 128);
                                mma_ts<MODE>(d, a, bhi, acc0);
                                mma_ts<MODE>(d, a, blo, 1u);
                                mma_ts<MODE>(d, a + 16, bhi, 1u);
                            } else {
                                mma_ts<MODE>(d, a, make_desc(st + bo, BN * 16, 128), acc0);
                            }
                        } else if (MODE == FDTD_N2F_BF16X3) {
                            const uint64_t ahi = make_desc(st + ao, BM * 16, 128);
                            const uint64_t alo = make_desc(st + C::A_BYTES + ao, BM * 16, 128);
                            const uint64_t bhi = make_desc(st + 2 * C::A_BYTES + bo, BN * 16, 128);
                            const uint64_t blo =
                                make_desc(st + 2 * C::A_BYTES + C::B_BYTES + bo, BN * 16, 128);
                            mma<MODE>(d, ahi, bhi, acc0);
                            mma<MODE>(d, ahi, blo, 1u);
                            mma<MODE>(d, alo, bhi, 1u);
                        } else {
                            const uint64_t a = make_desc(st + ao, BM * 16, 128);
                            const uint64_t bb = make_desc(st + C::A_BYTES + bo, BN * 16, 128);
                            mma<MODE>(d, a, bb, acc0);
                        }
                    }
                    mma_commit(smem_u32(&sm->empty[s]));
                    last = g;
                }
                if (!ok) break;
                mma_commit(smem_u32(&sm->acc_full[b]));
            }
            // MMAs complete in issue order, so the last commit covers all of them
            if (last >= 0) drain_bar(smem_u32(&sm->empty[last % NSTAGE]), (last / NSTAGE) & 1);
        }
    } else if ((warp >= 2 && warp < 6) || warp >= 10) {
        // group 0: warps 2-5; group h >= 1: warps 10 + 4(h-1) .. 13 + 4(h-1)
        // ---- A producers: phases u_p(o), one row (direction) per thread; NGRP
        // groups of four warps take the stages g with g % NGRP == group.
        // u_{ks*PS + i} = U_ks * w_i with w_i = e^{j2π γ i} (float, exact to an
        // ulp) and U_ks = e^{j2π γ ks PS}, evaluated in float64 at the group's
        // first stage of each n tile and advanced by a float64 rotation of NGRP K
        // steps after that, so each value carries one float rounding.
        const int grp = warp >= 10 ? 1 + (warp - 10) / 4 : 0;
        // ATM: the row is the TMEM lane this warp may write (lanes 32*(warp%4) ..)
        const int r = ATM ? 32 * (warp & 3) + lane
                          : (grp ? tid - (320 + 128 * (grp - 1)) : tid - 64);  // 0..127
        const int o = mt * BM + r;
        const bool valid = o < P.n_obs;
        const double gp = valid ? freq * F.pitch * P.dirs[3 * o + F.axis_p] / C0 : 0.0;
        float2 w[C::PS];
#pragma unroll
        for (int i = 0; i < C::PS; ++i) w[i] = phase_turns(gp, (double)i);
        const double2 W2 = zphase_turns(gp, (double)(NGRP * C::PS));
        // core-matrix offset of (row r, chunk c): (c*BM/8 + r/8)*128 + (r%8)*16
        const int roff = (r >> 3) * 128 + (r & 7) * 16;
        double2 U = make_double2(1.0, 0.0);
        int prev_ks = -1;
        for (int g = grp; g < total; g += NGRP) {
            const int s = g % NSTAGE, ks = g % KS;
            if (ks <= prev_ks || prev_ks < 0) U = zphase_turns(gp, (double)(ks * C::PS));
            prev_ks = ks;
            if (g >= NSTAGE) {
                bool free_ = wait_bar(smem_u32(&sm->empty[s]), ((g / NSTAGE) - 1) & 1, abort_flag,
                                      P.wait_ns);
                // ATM: the warp's tcgen05.st are warp-collective, so it leaves together
                if (ATM) free_ = __all_sync(0xffffffffu, free_);
                if (!free_) break;
                if (ATM) tc_fence_after();
            }
            unsigned char *st = stages + s * SSTAGE;
            const float2 uf = make_float2((float)U.x, (float)U.y);
            U = zmul(U, W2);
            float vals[2 * C::PS];
#pragma unroll
            for (int i = 0; i < C::PS; ++i) {
                const float2 u = cmul(uf, w[i]);
                vals[2 * i] = valid ? u.x : 0.f;
                vals[2 * i + 1] = valid ? u.y : 0.f;
            }
            if (ATM) {
                // one TMEM row: column c holds K = 2c, 2c+1 (BF16, hi then lo
                // 16 columns later) or K = c (TF32), the order of the smem rows
                const uint32_t ta = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + ATM_ACOL +
                                    (uint32_t)(s * 32);
                if (MODE == FDTD_N2F_BF16X3) {
                    uint32_t hr[16], lr[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(vals[2 * e], vals[2 * e + 1]);
                        const float2 hf = __bfloat1622float2(h);
                        const __nv_bfloat162 l =
                            __floats2bfloat162_rn(vals[2 * e] - hf.x, vals[2 * e + 1] - hf.y);
                        hr[e] = *reinterpret_cast<const uint32_t *>(&h);
                        lr[e] = *reinterpret_cast<const uint32_t *>(&l);
                    }
                    tmem_st16(ta, hr);
                    tmem_st16(ta + 16, lr);
                } else {
                    uint32_t t0[16], t1[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        t0[e] = __float_as_uint(tf32_rna(vals[e]));
                        t1[e] = __float_as_uint(tf32_rna(vals[16 + e]));
                    }
                    tmem_st16(ta, t0);
                    tmem_st16(ta + 16, t1);
                }
                tmem_st_wait();
                tc_fence_before();
            } else if (MODE == FDTD_N2F_BF16X3) {
#pragma unroll
                for (int c = 0; c < C::NCH; ++c) {
                    // packed conversions: two values per cvt.rn.bf16x2.f32
                    __align__(16) __nv_bfloat162 hi[4], lo[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float x0 = vals[8 * c + 2 * e], x1 = vals[8 * c + 2 * e + 1];
                        hi[e] = __floats2bfloat162_rn(x0, x1);
                        const float2 hf = __bfloat1622float2(hi[e]);
                        lo[e] = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
                    }
                    const int off = c * (BM / 8) * 128 + roff;
                    *reinterpret_cast<uint4 *>(st + off) = *reinterpret_cast<const uint4 *>(hi);
                    *reinterpret_cast<uint4 *>(st + C::A_BYTES + off) =
                        *reinterpret_cast<const uint4 *>(lo);
                }
            } else {
#pragma unroll
                for (int c = 0; c < C::NCH; ++c) {
                    float4 v4 = make_float4(tf32_rna(vals[4 * c]), tf32_rna(vals[4 * c + 1]),
                                            tf32_rna(vals[4 * c + 2]), tf32_rna(vals[4 * c + 3]));
                    *reinterpret_cast<float4 *>(st + c * (BM / 8) * 128 + roff) = v4;
                }
            }
            if (!ATM) fence_proxy_async();
            mbar_arrive(smem_u32(&sm->full_a[s]));
        }
    } else {
        // ---- epilogue: warps 6..9, one direction (TMEM lane) per thread; a warp
        // may read TMEM lanes 32*(warp % 4) .. +31 only
        const int q4 = warp & 3;
        const int row = q4 * 32 + lane;
        const int o = mt * BM + row;
        const bool valid = o < P.n_obs;
        double gq = 0.0, gc = 0.0;
        if (valid) {
            const double rn = P.dirs[3 * o + F.axis_n], rp = P.dirs[3 * o + F.axis_p],
                         rq = P.dirs[3 * o + F.axis_q];
            gq = freq * F.pitch * rq / C0;
            gc = freq * (rn * F.x_n + rp * F.o_p + rq * F.o_q) / C0;
        }
        // v_q = V_j * wq_i: V advanced by a float64 rotation per 4-sample chunk
        float2 wq[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) wq[i] = phase_turns(gq, (double)i);
        const double2 WQ = zphase_turns(gq, 4.0);
        double2 V = make_double2(1.0, 0.0);
        float2 S[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                       make_float2(0.f, 0.f)};
        for (int nt = 0; nt < NT; ++nt) {
            const int b = ATM ? 0 : (nt & 1);
            const uint32_t fpar = ATM ? (nt & 1) : ((nt >> 1) & 1);
            // tcgen05.ld is warp-collective: the warp leaves together on a timeout
            if (!__all_sync(0xffffffffu,
                            wait_bar(smem_u32(&sm->acc_full[b]), fpar, abort_flag, P.wait_ns)))
                break;
            tc_fence_after();
            const uint32_t base = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(b * BN);
#pragma unroll 1
            for (int j = 0; j < BN / 32; ++j) {
                float v[32];
                tmem_ld32(base + 32 * j, v);
                const float2 vf = make_float2((float)V.x, (float)V.y);
                V = zmul(V, WQ);
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) {
                    const float2 w = cmul(vf, wq[qq]);
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const float tr = v[(qq * 4 + c) * 2], ti = v[(qq * 4 + c) * 2 + 1];
                        S[c].x += w.x * tr - w.y * ti;
                        S[c].y += w.x * ti + w.y * tr;
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&sm->acc_empty[b]));
        }
        if (valid) {
            const float2 cph = phase_turns(gc, 1.0);
            float2 *out = P.partial + (((int64_t)fr * P.nfaces + fi) * P.n_obs + o) * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) out[c] = cmul(S[c], cph);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * BN);
    }
}

// Pack the currents of one face into the tiled B operand: for every (frequency,
// n tile, K step) a contiguous block [hi|lo][chunk NCH][256 rows][16 bytes]
// (BF16) or [chunk NCH][256 rows][16 bytes] (TF32), rows n = (q_local*4 + c)*2 + ri_n,
// K index k = 2p + ri_k, value Re/−Im/Im/Re of cur[p][q][c] by (ri_k, ri_n);
// zero outside [0, np) x [0, nq).
template <int MODE, typename CT>
__global__ void k_n2f_pack(const CT *cur, int nfreq, int np, int nq, int KS, int NT,
                           unsigned char *dst) {
    using C = Cfg<MODE>;
    constexpr int EPC = MODE == FDTD_N2F_BF16X3 ? 8 : 4;  // elements per 16-byte chunk
    const int64_t nchunks = (int64_t)nfreq * NT * KS * C::NCH * BN;
    for (int64_t q0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q0 < nchunks;
         q0 += (int64_t)gridDim.x * blockDim.x) {
        int64_t t = q0;
        const int row = (int)(t % BN);
        t /= BN;
        const int chunk = (int)(t % C::NCH);
        t /= C::NCH;
        const int ks = (int)(t % KS);
        t /= KS;
        const int nt = (int)(t % NT);
        const int fr = (int)(t / NT);
        const int ql = row >> 3, c = (row >> 1) & 3, ri_n = row & 1;
        const int q = nt * QT + ql;
        float vals[EPC];
#pragma unroll
        for (int e = 0; e < EPC; ++e) {
            const int k = ks * C::KR + chunk * EPC + e;
            const int p = k >> 1, ri_k = k & 1;
            float v = 0.f;
            if (p < np && q < nq) {
                const CT z = cur[(((int64_t)fr * np + p) * nq + q) * 4 + c];
                const float re = (float)z.x, im = (float)z.y;
                v = ri_k == 0 ? (ri_n == 0 ? re : im) : (ri_n == 0 ? -im : re);
            }
            vals[e] = v;
        }
        unsigned char *blk = dst + (((int64_t)fr * NT + nt) * KS + ks) * C::B_COPY;
        const int off = chunk * (BN / 8) * 128 + (row >> 3) * 128 + (row & 7) * 16;
        if (MODE == FDTD_N2F_BF16X3) {
            __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                hi[e] = __float2bfloat16_rn(vals[e]);
                lo[e] = __float2bfloat16_rn(vals[e] - __bfloat162float(hi[e]));
            }
            *reinterpret_cast<uint4 *>(blk + off) = *reinterpret_cast<const uint4 *>(hi);
            *reinterpret_cast<uint4 *>(blk + C::B_BYTES + off) = *reinterpret_cast<const uint4 *>(lo);
        } else {
            *reinterpret_cast<float4 *>(blk + off) =
                make_float4(tf32_rna(vals[0]), tf32_rna(vals[1]), tf32_rna(vals[2]), tf32_rna(vals[3]));
        }
    }
}

// NL[f][o][6] (complex64) = Σ_faces partial[f][face][o][c] mapped to (J_b, J_c, M_b, M_c).
__global__ void k_n2f_combine(Params P, int nfreq, float2 *nl) {
    const int64_t n = (int64_t)nfreq * P.n_obs;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int fr = (int)(q / P.n_obs), o = (int)(q % P.n_obs);
        float2 acc[6];
        for (int c = 0; c < 6; ++c) acc[c] = make_float2(0.f, 0.f);
        for (int fi = 0; fi < P.nfaces; ++fi) {
            const float2 *p = P.partial + (((int64_t)fr * P.nfaces + fi) * P.n_obs + o) * 4;
            for (int c = 0; c < 4; ++c) {
                const int m = P.comp_map[fi * 4 + c];
                acc[m].x += p[c].x;
                acc[m].y += p[c].y;
            }
        }
        for (int c = 0; c < 6; ++c) nl[q * 6 + c] = acc[c];
    }
}

// FP64 direct sum (no separation, no tensor cores): one block per (direction,
// frequency), exact phases e^{j2π f r̂·r'/c0} with the reduction in turns.
template <typename CT>
__global__ void k_n2f_fp64(Params P, double2 *nl) {
    const int o = blockIdx.x, fr = blockIdx.y;
    const double freq = P.freqs[fr];
    const double rv[3] = {P.dirs[3 * o], P.dirs[3 * o + 1], P.dirs[3 * o + 2]};
    double ar[6] = {0, 0, 0, 0, 0, 0}, ai[6] = {0, 0, 0, 0, 0, 0};
    for (int fi = 0; fi < P.nfaces; ++fi) {
        const Face &F = P.face[fi];
        const CT *cur = reinterpret_cast<const CT *>(P.cur[fi]) + (int64_t)fr * F.np * F.nq * 4;
        const double base = rv[F.axis_n] * F.x_n + rv[F.axis_p] * F.o_p + rv[F.axis_q] * F.o_q;
        const int64_t ns = (int64_t)F.np * F.nq;
        for (int64_t s = threadIdx.x; s < ns; s += blockDim.x) {
            const int p = (int)(s / F.nq), q = (int)(s % F.nq);
            double t = freq * (base + rv[F.axis_p] * F.pitch * p + rv[F.axis_q] * F.pitch * q) / C0;
            t = t - rint(t);
            double sn, cs;
            sincospi(2.0 * t, &sn, &cs);
            for (int c = 0; c < 4; ++c) {
                const CT z = cur[s * 4 + c];
                const int m = P.comp_map[fi * 4 + c];
                ar[m] += cs * (double)z.x - sn * (double)z.y;
                ai[m] += cs * (double)z.y + sn * (double)z.x;
            }
        }
    }
    __shared__ double red[2][6][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c = 0; c < 6; ++c) {
        double x = ar[c], y = ai[c];
        for (int sh = 16; sh > 0; sh >>= 1) {
            x += __shfl_down_sync(0xffffffffu, x, sh);
            y += __shfl_down_sync(0xffffffffu, y, sh);
        }
        if (lane == 0) {
            red[0][c][w] = x;
            red[1][c][w] = y;
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int c = threadIdx.x;
        double x = 0.0, y = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            x += red[0][c][i];
            y += red[1][c][i];
        }
        nl[((int64_t)fr * P.n_obs + o) * 6 + c] = make_double2(x, y);
    }
}

// ------------------------------------------------------------------- launchers
size_t stage_smem(int mode, bool atm) {
    size_t st;
    if (atm)
        st = (size_t)ATM_NST * (mode == FDTD_N2F_BF16X3 ? Cfg<FDTD_N2F_BF16X3>::B_COPY
                                                        : Cfg<FDTD_N2F_TF32>::B_COPY);
    else
        st = mode == FDTD_N2F_BF16X3
                 ? (size_t)Cfg<FDTD_N2F_BF16X3>::NST * Cfg<FDTD_N2F_BF16X3>::STAGE
                 : (size_t)Cfg<FDTD_N2F_TF32>::NST * Cfg<FDTD_N2F_TF32>::STAGE;
    return st + sizeof(Smem) + 64;
}

// Where the A operand lives: tensor memory by default; FDTD_B200_N2F_A=smem
// (read at each call) selects the shared-memory form, with the same MMAs in
// the same order.
bool a_in_tmem() {
    const char *e = getenv("FDTD_B200_N2F_A");
    return !(e && strcmp(e, "smem") == 0);
}

int b_copy_bytes(int mode) {
    return mode == FDTD_N2F_BF16X3 ? Cfg<FDTD_N2F_BF16X3>::B_COPY : Cfg<FDTD_N2F_TF32>::B_COPY;
}

int k_real_per_step(int mode) {
    return mode == FDTD_N2F_BF16X3 ? Cfg<FDTD_N2F_BF16X3>::KR : Cfg<FDTD_N2F_TF32>::KR;
}

template <typename CT>
cudaError_t launch_pack(int mode, const CT *cur, int nfreq, int np, int nq, int KS, int NT,
                        unsigned char *dst, cudaStream_t st) {
    const int nch = mode == FDTD_N2F_BF16X3 ? Cfg<FDTD_N2F_BF16X3>::NCH : Cfg<FDTD_N2F_TF32>::NCH;
    const int64_t n = (int64_t)nfreq * NT * KS * nch * BN;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (mode == FDTD_N2F_BF16X3)
        k_n2f_pack<FDTD_N2F_BF16X3, CT><<<(unsigned)blocks, 256, 0, st>>>(cur, nfreq, np, nq, KS, NT, dst);
    else
        k_n2f_pack<FDTD_N2F_TF32, CT><<<(unsigned)blocks, 256, 0, st>>>(cur, nfreq, np, nq, KS, NT, dst);
    count_launches(1);
    return cudaGetLastError();
}

namespace {
std::atomic<long long> g_wait_ns{(long long)WAIT_NS};
}

void set_wait_ns(int64_t ns) { g_wait_ns.store(ns < 0 ? (long long)WAIT_NS : ns); }

template <int MODE, bool ATM>
static cudaError_t launch_tc(const Params &P, int nfreq, cudaStream_t st) {
    const size_t smem = stage_smem(MODE, ATM);
    dim3 grid((P.n_obs + BM - 1) / BM, P.nfaces, nfreq);
    cudaError_t e =
        cudaFuncSetAttribute(k_n2f_tc<MODE, ATM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    k_n2f_tc<MODE, ATM><<<grid, NTHREADS, smem, st>>>(P);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_contract(int mode, const Params &Pin, int nfreq, cudaStream_t st) {
    Params P = Pin;
    P.wait_ns = (uint64_t)g_wait_ns.load();
    const bool atm = a_in_tmem();
    if (mode == FDTD_N2F_BF16X3)
        return atm ? launch_tc<FDTD_N2F_BF16X3, true>(P, nfreq, st)
                   : launch_tc<FDTD_N2F_BF16X3, false>(P, nfreq, st);
    return atm ? launch_tc<FDTD_N2F_TF32, true>(P, nfreq, st)
               : launch_tc<FDTD_N2F_TF32, false>(P, nfreq, st);
}

cudaError_t launch_combine(const Params &P, int nfreq, float2 *nl, cudaStream_t st) {
    const int64_t n = (int64_t)nfreq * P.n_obs;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_n2f_combine<<<(unsigned)blocks, 256, 0, st>>>(P, nfreq, nl);
    count_launches(1);
    return cudaGetLastError();
}

template <typename CT>
cudaError_t launch_fp64(const Params &P, int nfreq, double2 *nl, cudaStream_t st) {
    dim3 grid(P.n_obs, nfreq);
    k_n2f_fp64<CT><<<grid, 256, 0, st>>>(P, nl);
    count_launches(1);
    return cudaGetLastError();
}

int read_error(int reset) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_n2f_error, sizeof(int));
    if (reset) {
        int z = 0;
        cudaMemcpyToSymbol(g_n2f_error, &z, sizeof(int));
    }
    return v;
}

template cudaError_t launch_pack<float2>(int, const float2 *, int, int, int, int, int,
                                         unsigned char *, cudaStream_t);
template cudaError_t launch_pack<double2>(int, const double2 *, int, int, int, int, int,
                                          unsigned char *, cudaStream_t);
template cudaError_t launch_fp64<float2>(const Params &, int, double2 *, cudaStream_t);
template cudaError_t launch_fp64<double2>(const Params &, int, double2 *, cudaStream_t);

}  // namespace n2f
}  // namespace fdtd
