// The spectral-mode print kernel: the print stage (negative density -> linear output RGB) with a chosen
// arithmetic for its two spectral integrals, R_k = sum_l 10^-(d . eps(l) + beta(l)) wt_k(l) (reference
// kernels/print.metal:165-189), at 81 or up to SPKB_NL_MAX wavelengths. The stages around the integrals
// are the print kernel's (print_common.cuh).
//
// One pixel per thread, 128-pixel tiles, persistent CTAs.
//
// Tensor-core modes (tcgen05): per integral the wavelengths go in chunks of 16. Each thread forms
// T(l) = 2^(sum_c d_c e_c(l)) for its pixel on the CUDA cores (the print kernel's binary32 operations) and
// writes its row of the A operand (128 pixels x 16 wavelengths: the thread's pixel is its tensor-memory
// lane, the wavelengths consecutive 32-bit columns) into one of three tensor-memory stages with
// tcgen05.st: bf16(T) (BF16), bf16(T) and bf16(T - bf16(T)) in the next 8 columns (BF16X3), or T in
// binary32 (TF32, of which the tensor core reads the TF32 part). One thread then issues the chunk's MMAs
// with A from tensor memory, D[128 x 16] (+)= A B^T with B the pass's 16-row weight table in shared memory
// (rows 0..2 the weights' BF16 high parts, rows 3..5 their low parts), accumulating in tensor memory, and
// commits them to the stage's mbarrier, which releases the stage for the chunk three later. Tensor memory:
// 64 columns per CTA, D in columns 0..15, the stages from column 16. After the last chunk each thread reads
// its pixel's row of D (tcgen05.ld): R_k = D[k] + D[k + 3] for BF16X3 (all four products of the hi and lo
// parts), R_k = D[k] otherwise.
//
// CUDA-core modes: F32 performs the print kernel's binary32 operations in its order (at the resources' 81
// wavelengths the output equals k_print's bit for bit); F64 evaluates both integrals in binary64 from the
// binary64 tables.
//
// Every mbarrier wait gives up after 4e9 SM clocks (about 2 s; a test hook can shorten the stage waits'
// limit to a few clocks so that one runs out). A wait that gives up is made known to the whole CTA at the
// chunk's barrier; from then on the CTA forms no operands, issues no MMAs and reads no tensor memory, leaves
// its tile loop at the tile's end, waits for the MMAs it already issued (bounded by the full limit, never
// the shortened one), frees its tensor memory and sets *err.
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>

#include "../kernel_args.h"
#include "launch.hpp"
#include "print_common.cuh"

namespace spkb::dev {

namespace {

constexpr uint32_t kTcThreads = 128;  // the MMA's M: one pixel per thread and per TMEM lane
constexpr uint32_t kChunk = 16;       // wavelengths per A stage
constexpr uint32_t kStages = 3;
constexpr uint32_t kTmemCols = 64;    // D in columns 0..15, the A stages in 16..63
constexpr uint32_t kStageCols = 16;   // one A stage: 16 wavelengths of 32 bits (TF32), or BF16 hi and lo halves
constexpr long long kWaitCycles = 4000000000ll;

// instruction descriptors: D binary32 (bits 4-5 = 1), A and B format (bits 7-9, 10-12: 1 BF16, 2 TF32),
// both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24; N = 16, M = 128
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__host__ __device__ constexpr bool tc_mode(int m) {
    return m == SPKB_SPEC_TF32 || m == SPKB_SPEC_BF16 || m == SPKB_SPEC_BF16X3;
}
__host__ __device__ constexpr uint32_t elem_bytes(int m) { return m == SPKB_SPEC_TF32 ? 4u : 2u; }
__host__ __device__ constexpr uint32_t round_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// Dynamic shared memory of one CTA: the binary64 tables (mode F64), the B tiles of the tensor-core modes,
// then the mbarriers (kStages stage barriers and a teardown barrier) and the tensor-memory address slot.
struct SmemLayout {
    uint32_t e, w, e64, w64, b, bar, total;
};
// At more than 96 wavelengths the spectral loops stay rolled; the binary32 CUDA-core path then reads its
// tables from shared memory (a constant-bank operand needs a fixed index), the tensor-core paths keep them
// in the constant bank (indexed loads, no shared memory taken from the CTAs' stages).
__host__ __device__ constexpr bool tables_in_smem(int m, uint32_t nl_pad) { return m == SPKB_SPEC_F32 && nl_pad > 96; }
__host__ __device__ constexpr SmemLayout smem_layout(int m, uint32_t nl_pad) {
    SmemLayout L{};
    uint32_t off = 0;
    L.e = off;
    if (tables_in_smem(m, nl_pad)) off = round_up(off + 2 * (nl_pad / 2) * 32, 128);
    L.w = off;
    if (tables_in_smem(m, nl_pad)) off = round_up(off + 2 * nl_pad * 16, 128);
    L.e64 = off;
    if (m == SPKB_SPEC_F64) off = round_up(off + 2 * nl_pad * 32, 128);
    L.w64 = off;
    if (m == SPKB_SPEC_F64) off = round_up(off + 2 * nl_pad * 32, 128);
    L.b = off;
    if (tc_mode(m)) off = round_up(off + 2 * 16 * nl_pad * elem_bytes(m), 128);
    L.bar = off;
    off += 8 * (kStages + 1) + 8;
    L.total = round_up(off, 128);
    return L;
}

// Kernel parameters (constant bank, up to 28 KB): the frame's print arguments and the binary32
// per-wavelength tables, so that the unrolled spectral loops take their table operands from the constant
// bank as the print kernel does.
template <int NLP>
struct alignas(16) SpectralParams {
    PrintArgs a;
    float e[2][NLP / 2][6];  // [pass][l / 2] = {e0(l), e0(l+1), e1(l), e1(l+1), e2(l), e2(l+1)}
    float w[2][NLP][3];      // [pass][l] = w_k(l), binary32 (mode F32)
    const SpectralTablesN* tab;  // device: the B tiles and the binary64 tables
    const float* neg;
    float* rgb;
    float* contraction;
    uint32_t* err;
    long long wait_limit;  // SM clocks a stage wait may take before it gives up
    uint32_t n, nl;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// the phase's completion tested without waiting
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for the completion of the barrier's phase of the given parity; false after `limit` SM clocks
// (kWaitCycles: about 2 s at the B200's clocks). The clock is read only once the phase was found incomplete.
// try_wait may suspend the thread for a while by itself, so a shortened limit (the test hook) polls with
// the non-blocking test_wait instead, and a phase still running then runs the wait out at once.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
    if (limit < kWaitCycles) {
        const long long t0 = clock64();
        for (;;) {
            if (mbar_test(bar, parity)) return true;
            if (clock64() - t0 > limit) return false;
        }
    }
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (clock64() - t0 > limit) return false;
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(cols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// this thread's generic-proxy writes to shared memory become visible to the tensor cores' (async) proxy
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (+)= A B^T with A in tensor memory (a: the tile's column address, lane 0) and B in shared memory
__device__ __forceinline__ void mma_bf16(uint32_t d, uint32_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(b), "r"(kIdescBf16), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_tf32(uint32_t d, uint32_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(b), "r"(kIdescTf32), "r"(acc)
        : "memory");
}
// this thread's 8 consecutive 32-bit columns of its lane, from the column address taddr (the warp's 32
// lanes start at taddr's lane field); tmem_wait_st waits for this thread's stores to complete
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t r[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// the barrier's arrival once every MMA this thread issued before it has completed
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// columns 0..7 of this thread's TMEM lane (the warp's 32 lanes start at taddr's lane field)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float v[8]) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// shared-memory matrix descriptor, no swizzle: start, leading (K-direction core-matrix) and stride
// (8-row group) byte offsets, each >> 4; descriptor version 1 at bit 46
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// bf16 pair {lo in the low half, hi in the high half}, round to nearest even
__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}


__device__ __forceinline__ void copy16(unsigned char* dst, const void* src, uint32_t bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (uint32_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
}

// the upper halves of two binary32 values: their BF16 truncations {lo in the low half, hi in the high half}
__device__ __forceinline__ uint32_t upper_halves(float lo, float hi) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, 0x7632;" : "=r"(r) : "r"(__float_as_uint(lo)), "r"(__float_as_uint(hi)));
    return r;
}

// T(l) = 2^(sum_c d_c e_c(l)) of this thread's pixel for wavelengths l0 .. l0 + 7
// (tables from the kernel parameters, or from shared memory: smem_e, [pass][l / 2][8])
template <int NLP, uint32_t PASS, bool SMEM>
__device__ __forceinline__ void transmittance8(const SpectralParams<NLP>& p, const float* smem_e, uint32_t l0,
                                               float2 D0, float2 D1, float2 D2, float T[8]) {
#pragma unroll
    for (uint32_t i = 0; i < 4; ++i) {
        float2 e0, e1, e2;
        if constexpr (SMEM) {
            const float* ep = smem_e + (PASS * (NLP / 2) + l0 / 2 + i) * 8;
            const float4 a = *reinterpret_cast<const float4*>(ep);
            e0 = make_float2(a.x, a.y);
            e1 = make_float2(a.z, a.w);
            e2 = *reinterpret_cast<const float2*>(ep + 4);
        } else {
            const float* ep = p.e[PASS][l0 / 2 + i];
            e0 = make_float2(ep[0], ep[1]);
            e1 = make_float2(ep[2], ep[3]);
            e2 = make_float2(ep[4], ep[5]);
        }
        const float2 e = __ffma2_rn(D2, e2, __ffma2_rn(D1, e1, __fmul2_rn(D0, e0)));
        T[2 * i] = ex2_ftz(e.x);
        T[2 * i + 1] = ex2_ftz(e.y);
    }
}

// T over wavelengths j*kChunk .. j*kChunk + kChunk - 1 for this thread's pixel, into its lane of the A stage
// at tensor-memory column address `stage` (the warp's lanes):
//   TF32    T (binary32), columns 0..15;
//   BF16    bf16(T), rounded to nearest, wavelength pairs in columns 0..7 (the lower wavelength in the low half);
//   BF16X3  hi = T truncated to BF16 in columns 0..7 and lo = bf16(T - hi) in columns 8..15 (T - hi is exact
//           in binary32).
template <int M, int NLP, uint32_t PASS>
__device__ __forceinline__ void produce(const SpectralParams<NLP>& p, const float* smem_e, uint32_t j, float2 D0,
                                        float2 D1, float2 D2, uint32_t stage) {
    uint32_t h[kChunk / 2], l[kChunk / 2];
#pragma unroll
    for (uint32_t q = 0; q < kChunk / 8; ++q) {
        float T[8];
        transmittance8<NLP, PASS, false>(p, smem_e, j * kChunk + q * 8, D0, D1, D2, T);
        if constexpr (M == SPKB_SPEC_TF32) {
            uint32_t t[8];
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i) t[i] = __float_as_uint(T[i]);
            tmem_st8(stage + 8 * q, t);
        } else {
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                const float a = T[2 * i], b = T[2 * i + 1];
                if constexpr (M == SPKB_SPEC_BF16) {
                    h[4 * q + i] = bf16x2(a, b);
                } else {
                    h[4 * q + i] = upper_halves(a, b);
                    // T - hi = T + (-1) hi, exact
                    const float2 hi2 = make_float2(__uint_as_float(__float_as_uint(a) & 0xFFFF0000u),
                                                   __uint_as_float(__float_as_uint(b) & 0xFFFF0000u));
                    const float2 rem = __ffma2_rn(hi2, make_float2(-1.0f, -1.0f), make_float2(a, b));
                    l[4 * q + i] = bf16x2(rem.x, rem.y);
                }
            }
        }
    }
    if constexpr (M != SPKB_SPEC_TF32) tmem_st8(stage, h);
    if constexpr (M == SPKB_SPEC_BF16X3) tmem_st8(stage + 8, l);
}

// the MMAs of chunk j: A the stage at tensor-memory column address a_tmem, B the pass's table at b_saddr
// (16 x NLP)
template <int M, int NLP>
__device__ __forceinline__ void issue(uint32_t tmem, uint32_t a_tmem, uint32_t b_saddr, uint32_t j) {
    if constexpr (M == SPKB_SPEC_TF32) {
        constexpr uint32_t sbo_b = (NLP * 4 / 16) * 128;
#pragma unroll
        for (uint32_t s = 0; s < kChunk / 8; ++s) {  // K = 8 per MMA: 8 columns
            const uint64_t b = smem_desc(b_saddr + (j * (kChunk * 4 / 16) + 2 * s) * 128, 128, sbo_b);
            mma_tf32(tmem, a_tmem + 8 * s, b, (j | s) != 0);
        }
    } else {
        constexpr uint32_t sbo_b = (NLP * 2 / 16) * 128;
        const uint64_t b = smem_desc(b_saddr + j * (kChunk * 2 / 16) * 128, 128, sbo_b);  // K = 16 per MMA
        mma_bf16(tmem, a_tmem, b, j != 0);
        if constexpr (M == SPKB_SPEC_BF16X3) mma_bf16(tmem, a_tmem + 8, b, 1u);
    }
}

// One integral on the tensor cores for the CTA's 128 pixels. g counts the CTA's chunks (stage and
// barrier phase); ok, the same in every thread of the CTA, turns false once any thread's wait gave up:
// from then on nothing is produced, issued, waited for or read from tensor memory (R is 0).
template <int M, int NLP, uint32_t PASS>
__device__ __forceinline__ void contract_tc(const SpectralParams<NLP>& p, unsigned char* smem, uint32_t tmem,
                                            const float d[3], float R[3], uint32_t& g, bool& ok) {
    constexpr SmemLayout L = smem_layout(M, NLP);
    const uint32_t tid = threadIdx.x;
    const uint32_t lanes = (32u * (tid / 32u)) << 16;  // this warp's 32 lanes
    const float2 D0 = make_float2(d[0], d[0]), D1 = make_float2(d[1], d[1]), D2 = make_float2(d[2], d[2]);
    const uint32_t b_saddr = smem_addr(smem + L.b) + PASS * 16 * NLP * elem_bytes(M);
    const uint32_t bar0 = smem_addr(smem + L.bar);
    // unrolled at 81 wavelengths (table operands from the constant bank); at 401 the loop stays rolled,
    // its code would not fit the instruction cache
    constexpr int kUnroll = NLP <= 96 ? int(NLP / kChunk) : 1;
#pragma unroll kUnroll
    for (uint32_t j = 0; j < NLP / kChunk; ++j, ++g) {
        const uint32_t st = g % kStages;
        const uint32_t stage = tmem + 16u + st * kStageCols;
        // the MMAs of chunk g - kStages read this stage
        bool mine = ok;
        if (g >= kStages && mine) mine = mbar_wait(bar0 + 8 * st, ((g / kStages) - 1) & 1u, p.wait_limit);
        if (mine) {
            tc_fence_after();
            produce<M, NLP, PASS>(p, reinterpret_cast<const float*>(smem + L.e), j, D0, D1, D2, stage + lanes);
            tmem_wait_st();
        }
        tc_fence_before();
        ok = __syncthreads_or(mine ? 0 : 1) == 0;
        if (tid == 0 && ok) {
            tc_fence_after();
            issue<M, NLP>(tmem, stage, b_saddr, j);
            mma_commit(bar0 + 8 * st);
        }
    }
    const uint32_t last = g - 1;
    bool mine = ok;
    if (mine) mine = mbar_wait(bar0 + 8 * (last % kStages), (last / kStages) & 1u, p.wait_limit);
    ok = __syncthreads_or(mine ? 0 : 1) == 0;  // uniform: tcgen05.ld is warp-collective
    if (!ok) {
        R[0] = R[1] = R[2] = 0.0f;
        return;
    }
    tc_fence_after();
    float v[8];
    tmem_ld8(tmem + lanes, v);
#pragma unroll
    for (int k = 0; k < 3; ++k) R[k] = M == SPKB_SPEC_BF16X3 ? v[k] + v[k + 3] : v[k];
}

// One integral on the CUDA cores in binary32: the print kernel's operations, wavelength pairs ascending
template <int NLP, uint32_t PASS>
__device__ __forceinline__ void contract_f32(const SpectralParams<NLP>& p, const unsigned char* smem, const float d[3],
                                             float R[3]) {
    constexpr SmemLayout L = smem_layout(SPKB_SPEC_F32, NLP);
    const float* smem_e = reinterpret_cast<const float*>(smem + L.e);
    const float* smem_w = reinterpret_cast<const float*>(smem + L.w) + PASS * NLP * 4;
    const float2 D0 = make_float2(d[0], d[0]), D1 = make_float2(d[1], d[1]), D2 = make_float2(d[2], d[2]);
    float r0 = 0.0f, r1 = 0.0f, r2 = 0.0f;
    constexpr int kUnroll = NLP <= 96 ? int(NLP / 8) : 1;
#pragma unroll kUnroll
    for (uint32_t l0 = 0; l0 < NLP; l0 += 8) {
        if (l0 >= p.nl) break;
        float T[8];
        transmittance8<NLP, PASS, tables_in_smem(SPKB_SPEC_F32, NLP)>(p, smem_e, l0, D0, D1, D2, T);
#pragma unroll
        for (uint32_t i = 0; i < 8; ++i) {
            // past nl the weights are zero: fma(T, 0, r) = r
            float w0, w1, w2;
            if constexpr (tables_in_smem(SPKB_SPEC_F32, NLP)) {
                const float4 w = *reinterpret_cast<const float4*>(smem_w + (l0 + i) * 4);
                w0 = w.x;
                w1 = w.y;
                w2 = w.z;
            } else {
                w0 = p.w[PASS][l0 + i][0];
                w1 = p.w[PASS][l0 + i][1];
                w2 = p.w[PASS][l0 + i][2];
            }
            r0 = fmaf(T[i], w0, r0);
            r1 = fmaf(T[i], w1, r1);
            r2 = fmaf(T[i], w2, r2);
        }
    }
    R[0] = r0;
    R[1] = r1;
    R[2] = r2;
}

// One integral in binary64 from the binary64 tables; the sums return rounded to binary32
__device__ __forceinline__ void contract_f64(const double* __restrict__ E, const double* __restrict__ W, uint32_t nl,
                                             const float d[3], float R[3]) {
    const double a0 = d[0], a1 = d[1], a2 = d[2];
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    for (uint32_t l = 0; l < nl; ++l) {
        const double* e = E + 4 * l;
        const double* w = W + 4 * l;
        const double T = exp2(fma(a2, e[2], fma(a1, e[1], a0 * e[0])));
        r0 = fma(T, w[0], r0);
        r1 = fma(T, w[1], r1);
        r2 = fma(T, w[2], r2);
    }
    R[0] = float(r0);
    R[1] = float(r1);
    R[2] = float(r2);
}

template <int M, int NLP, uint32_t PASS>
__device__ __forceinline__ void contract(const SpectralParams<NLP>& p, unsigned char* smem, uint32_t tmem,
                                         const float d[3], float R[3], uint32_t& g, bool& ok) {
    if constexpr (tc_mode(M)) {
        contract_tc<M, NLP, PASS>(p, smem, tmem, d, R, g, ok);
    } else if constexpr (M == SPKB_SPEC_F32) {
        contract_f32<NLP, PASS>(p, smem, d, R);
    } else {
        constexpr SmemLayout L = smem_layout(M, NLP);
        contract_f64(reinterpret_cast<const double*>(smem + L.e64) + PASS * NLP * 4,
                     reinterpret_cast<const double*>(smem + L.w64) + PASS * NLP * 4, p.nl, d, R);
    }
}

template <int M, int NLP>
__global__ void __launch_bounds__(kTcThreads) k_print_spectral(const __grid_constant__ SpectralParams<NLP> p) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr bool kTc = tc_mode(M);
    constexpr SmemLayout L = smem_layout(M, NLP);
    const uint32_t tid = threadIdx.x;
    const SpectralTablesN* tab = p.tab;
    for (uint32_t q = 0; q < 2; ++q) {
        if constexpr (tables_in_smem(M, NLP)) {
            copy16(smem + L.e + q * (NLP / 2) * 32, tab->e_pairs[q], (NLP / 2) * 32);
            copy16(smem + L.w + q * NLP * 16, tab->w[q], NLP * 16);
        }
        if constexpr (M == SPKB_SPEC_F64) {
            copy16(smem + L.e64 + q * NLP * 32, tab->e64[q], NLP * 32);
            copy16(smem + L.w64 + q * NLP * 32, tab->w64[q], NLP * 32);
        }
        if constexpr (M == SPKB_SPEC_TF32) copy16(smem + L.b + q * 16 * NLP * 4, tab->b_tf32[q], 16 * NLP * 4);
        if constexpr (M == SPKB_SPEC_BF16 || M == SPKB_SPEC_BF16X3)
            copy16(smem + L.b + q * 16 * NLP * 2, tab->b_bf16[q], 16 * NLP * 2);
    }
    const uint32_t bar0 = smem_addr(smem + L.bar);
    const uint32_t bar_end = bar0 + 8 * kStages;
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + L.bar + 8 * (kStages + 1));
    if constexpr (kTc) {
        if (tid == 0) {
            for (uint32_t s = 0; s <= kStages; ++s) mbar_init(bar0 + 8 * s, 1);
            fence_mbar_init();
        }
        if (tid < 32) {
            tmem_alloc(smem_addr(slot), kTmemCols);
            tmem_relinquish();
        }
        fence_async_smem();  // the B tiles, written above, are read by the tensor cores
        tc_fence_before();
    }
    __syncthreads();
    uint32_t tmem = 0;
    if constexpr (kTc) {
        tc_fence_after();
        tmem = *slot;
    }
    const PrintArgs& a = p.a;
    const uint32_t n = p.n;

    uint32_t g = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; size_t(tile) * kTcThreads < n; tile += gridDim.x) {
        const uint32_t px = tile * kTcThreads + tid;
        const bool valid = px < n;
        float d[3] = {0.0f, 0.0f, 0.0f};
        if (valid) {
            d[0] = p.neg[3 * size_t(px)];
            d[1] = p.neg[3 * size_t(px) + 1];
            d[2] = p.neg[3 * size_t(px) + 2];
        }
        float R[3];
        if (a.printed) {
            contract<M, NLP, 0>(p, smem, tmem, d, R, g, ok);
            if (p.contraction && valid) {
                p.contraction[3 * size_t(px)] = R[0];
                p.contraction[3 * size_t(px) + 1] = R[1];
                p.contraction[3 * size_t(px) + 2] = R[2];
            }
#pragma unroll
            for (uint32_t c = 0; c < 3; ++c) d[c] = print_density(a, c, R[c]);
        }
        contract<M, NLP, 1>(p, smem, tmem, d, R, g, ok);
        if (valid) {
            float x = fmaxf(R[0], 0.0f) + kTiny;
            float y = fmaxf(R[1], 0.0f) + kTiny;
            float z = fmaxf(R[2], 0.0f) + kTiny;
            apply_levels(a, x, y, z);
            add_glare(a, size_t(px), x, y, z);
            float r, gg, b;
            mat_apply(a.to_rgb, x, y, z, r, gg, b);
            gamut(a, r, gg, b);
            float* o = p.rgb + 3 * size_t(px);
            o[0] = r;
            o[1] = gg;
            o[2] = b;
        }
        if constexpr (kTc) {
            if (__syncthreads_or(ok ? 0 : 1)) break;
        }
    }

    if constexpr (kTc) {
        tc_fence_before();
        __syncthreads();
        bool done = true;
        if (tid == 0) {
            mma_commit(bar_end);
            done = mbar_wait(bar_end, 0, kWaitCycles);  // every issued MMA ends before the tensor memory is freed
        }
        const int failed = __syncthreads_or((ok && done) ? 0 : 1);
        if (tid < 32) {
            tc_fence_after();
            tmem_dealloc(tmem, kTmemCols);
        }
        if (tid == 0 && failed) atomicOr(p.err, 1u);
    }
}

long long g_wait_limit = 0;  // spkx_test_set_tc_wait_limit: 0 the full limit

template <int M, int NLP>
void launch_spectral(const PrintArgs& a, const SpectralTablesN& host_tab, const SpectralTablesN* tab, const float* neg,
                     float* rgb, uint32_t n, float* contraction, uint32_t* err, cudaStream_t s) {
    // a tensor-core CTA takes at least 25 KB of shared memory, so that no more than 8 are resident on an SM:
    // with 64 tensor-memory columns each, 8 fill the SM's 512, and a ninth would wait in tcgen05.alloc
    constexpr uint32_t smem = tc_mode(M) && smem_layout(M, NLP).total < 25u * 1024u ? 25u * 1024u
                                                                                 : smem_layout(M, NLP).total;
    auto kernel = k_print_spectral<M, NLP>;
    ensure_smem(reinterpret_cast<const void*>(kernel), int(smem));
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared));
    auto prm = std::make_unique<SpectralParams<NLP>>();
    prm->a = a;
    for (uint32_t q = 0; q < 2; ++q) {
        for (uint32_t l = 0; l < NLP; ++l)
            for (uint32_t c = 0; c < 3; ++c) {
                prm->e[q][l / 2][2 * c + (l & 1)] = host_tab.e_pairs[q][l / 2][2 * c + (l & 1)];
                prm->w[q][l][c] = host_tab.w[q][l][c];
            }
    }
    prm->tab = tab;
    prm->neg = neg;
    prm->rgb = rgb;
    prm->contraction = contraction;
    prm->err = err;
    prm->wait_limit = g_wait_limit > 0 ? g_wait_limit : kWaitCycles;
    prm->n = n;
    prm->nl = host_tab.nl;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTcThreads, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        per_sm = 0;
    }
    // resident CTAs by shared memory (228 KB per SM, 1 KB reserved per CTA), threads (2048 per SM) and, in
    // the tensor-core modes, tensor memory (512 columns per SM); a CTA beyond the resident ones only starts
    // later, no CTA waits on another
    const int by_smem = int((228u * 1024u) / (smem + 1024u));
    const int fit = by_smem < 16 ? by_smem : 16;
    if (per_sm < fit) per_sm = fit;
    if (tc_mode(M) && per_sm > int(512u / kTmemCols)) per_sm = int(512u / kTmemCols);
    static_assert(512u / kTmemCols == 8u, "the shared-memory floor above holds 8 CTAs per SM");
    const uint64_t tiles = (uint64_t(n) + kTcThreads - 1) / kTcThreads;
    const uint64_t resident = uint64_t(sms > 0 ? sms : 1) * uint64_t(per_sm > 0 ? per_sm : 1);
    const uint32_t grid = uint32_t(tiles < resident ? tiles : resident);
    kernel<<<grid, kTcThreads, smem, s>>>(*prm);
}

template <int M>
void launch_mode(const PrintArgs& a, const SpectralTablesN& host_tab, const SpectralTablesN* tab, const float* neg,
                 float* rgb, uint32_t n, float* contraction, uint32_t* err, cudaStream_t s) {
    if (host_tab.nl_pad == 96) launch_spectral<M, 96>(a, host_tab, tab, neg, rgb, n, contraction, err, s);
    else launch_spectral<M, SPKB_NL_MAX>(a, host_tab, tab, neg, rgb, n, contraction, err, s);
}

}  // namespace

bool print_spectral_supported(uint32_t nl_pad) { return nl_pad == 96 || nl_pad == SPKB_NL_MAX; }

void set_tc_wait_limit(long long cycles) { g_wait_limit = cycles; }

void print_spectral(const PrintArgs& a, const SpectralTablesN& host_tab, const SpectralTablesN* tab, int mode,
                    const float* neg, float* rgb, uint32_t n, float* contraction, uint32_t* err, cudaStream_t s) {
    if (n == 0) return;
    Probe p("print_spectral", s);
    switch (mode) {
        case SPKB_SPEC_F32: launch_mode<SPKB_SPEC_F32>(a, host_tab, tab, neg, rgb, n, contraction, err, s); break;
        case SPKB_SPEC_F64: launch_mode<SPKB_SPEC_F64>(a, host_tab, tab, neg, rgb, n, contraction, err, s); break;
        case SPKB_SPEC_TF32: launch_mode<SPKB_SPEC_TF32>(a, host_tab, tab, neg, rgb, n, contraction, err, s); break;
        case SPKB_SPEC_BF16: launch_mode<SPKB_SPEC_BF16>(a, host_tab, tab, neg, rgb, n, contraction, err, s); break;
        default: launch_mode<SPKB_SPEC_BF16X3>(a, host_tab, tab, neg, rgb, n, contraction, err, s); break;
    }
}

}  // namespace spkb::dev
