// Recursive Gaussian blurs (Young and van Vliet, third order) over whole lines held in shared memory,
// evaluated block-parallel.
//
// The recurrence of one line (reference kernels/fx_blur.metal:125-170):
//   forward   w[i] = B x[i] + B1 w[i-1] + B2 w[i-2] + B3 w[i-3],  w[-1] = w[-2] = w[-3] = x[0];  u[i] = float(w[i])
//   backward  y[i] = B u[i] + B1 y[i+1] + B2 y[i+2] + B3 y[i+3],  y[n] = y[n+1] = y[n+2] = u[n-1]
// is a linear time-invariant system, so a line cut into segments of L samples can be solved in three
// steps (the block decomposition of Nehab, Maximo, Lima and Hoppe, "GPU-efficient recursive filtering
// and summed-area tables", SIGGRAPH Asia 2011):
//   1. every segment runs the recurrence from a zero state (the first segment from the true edge
//      state) and keeps its last three values e_s;
//   2. the true state entering segment s+1 is S_s = e_s + M S_{s-1}, with M the 3 x 3 map of an
//      entry state through L steps of the homogeneous recurrence (a parallel scan over the segments);
//   3. every segment recomputes from its true entry state and stores its values.
// State and the carries are binary64 (the reference keeps double-float state on its GPU and double
// state on its host copy); x, u and y are stored as binary32 exactly as there.
//
// k_iir_rows: one CTA per image row, 3 lines x kSegRows segments; the row (3 w floats) in shared memory,
//             loaded afresh for every mixture component, blurred and written to the component's plane.
// k_iir_cols: one CTA per strip of 4 pixel columns (12 lines); every component's row result blurred
//             down the columns in turn; the mixture accumulated as the reference's fused passes do
//             (acc = 0 + w0 y0, acc = acc + w_k y_k) and the halation mix raw := a raw + b acc written
//             in place of raw; a plain blur (one component) stores its lines as they are.
//             A full strip (frame width a multiple of 4) comes into shared memory by TMA: the component's
//             plane is a 2-D tensor (3 w floats x h rows), and the strip is a column of 12-float boxes of up
//             to 256 rows, all completing on one mbarrier. Its waits are bounded: one that gives up counts
//             itself (g_iir_gave_up), waits again under the full limit for the copies in flight, and if
//             even they never land the CTA loads this and every later strip with plain copies.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>

#include "../kernel_args.h"
#include "iir.hpp"

namespace spkb::dev {

namespace {

#ifndef SPKB_IIR_SEG_ROWS
#define SPKB_IIR_SEG_ROWS 64
#endif
constexpr int kSegRows = SPKB_IIR_SEG_ROWS;  // segments per channel line in a row (4K rows: 0.185 ms at 128, 0.152 at 64)
static_assert(kSegRows <= (1 << kIirScanSteps), "the carry scan composes at most 2^kIirScanSteps segments");
constexpr int kRowThreads = 3 * kSegRows;
constexpr int kColPixels = 4;       // pixels per column strip
constexpr int kColLines = 3 * kColPixels;
#ifndef SPKB_IIR_SEG_COLS
#define SPKB_IIR_SEG_COLS 32
#endif
constexpr int kSegCols = SPKB_IIR_SEG_COLS;  // segments per column line (32: two 4K strips per SM)
static_assert(kSegCols <= (1 << kIirScanSteps), "the carry scan composes at most 2^kIirScanSteps segments");
constexpr int kColThreads = kColLines * kSegCols;

// The column pass's tensor maps, one per component plane, and the strip's box geometry: `boxes` boxes of
// `box_rows` rows (a multiple of 8, at most 256) cover the frame's rows; the strip buffer holds
// boxes * box_rows rows, and the rows past the frame are zero-filled by the copy and never read.
struct IirColMaps {
    CUtensorMap map[SPKB_MAX_COMPONENTS];
    long long wait_limit;  // SM clocks a strip wait may take before it gives up
    uint32_t box_rows, boxes;
    uint32_t use_tma;      // 0: plain copies (a width that is not a multiple of 4, or no tensor map)
};

#ifndef SPKB_IIR_COL_TMA
#define SPKB_IIR_COL_TMA 1
#endif
constexpr bool kColTma = SPKB_IIR_COL_TMA != 0;  // 0: every strip by plain 16-byte copies

constexpr long long kWaitCycles = 4000000000LL;  // about 2 s at the B200's clocks
__device__ unsigned int g_iir_gave_up;           // strip waits that gave up, since the last read

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// this thread's earlier shared-memory accesses ordered before the asynchronous (TMA) proxy's next ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

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

// the barrier's phase of the given parity completed; false once `limit` SM clocks have passed without it.
// try_wait may suspend the thread for a while by itself, so a shortened limit (the test hook) polls with
// the non-blocking test_wait instead.
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

// one box of a 2-D tensor map at element coordinates (x, y) into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

struct Coef {
    double B, B1, B2, B3;
};

__device__ __forceinline__ double step(const Coef& k, double x, double s1, double s2, double s3) {
    // the oldest state first and the newest last: each state is j steps old when it enters the j-th
    // multiply-add from the end, so the chain costs one multiply-add latency per sample
    return fma(k.B1, s1, fma(k.B2, s2, fma(k.B3, s3, k.B * x)));
}

// Forward pass over one segment [a, b) of a line in shared memory (element i at base[i * stride]).
// Zero-state run: returns the end state. Writing run: from `in` state, stores float(w) back.
__device__ __forceinline__ void seg_forward(const Coef& k, float* base, int stride, int a, int b, double& s1,
                                            double& s2, double& s3, bool write) {
#pragma unroll 4
    for (int i = a; i < b; ++i) {
        const double t = step(k, double(base[i * stride]), s1, s2, s3);
        s3 = s2;
        s2 = s1;
        s1 = t;
        if (write) base[i * stride] = float(t);
    }
}

__device__ __forceinline__ void seg_backward(const Coef& k, float* base, int stride, int a, int b, double& s1,
                                             double& s2, double& s3, bool write) {
#pragma unroll 4
    for (int i = b - 1; i >= a; --i) {
        const double t = step(k, double(base[i * stride]), s1, s2, s3);
        s3 = s2;
        s2 = s1;
        s1 = t;
        if (write) base[i * stride] = float(t);
    }
}

// The true entry states of the segments, by a Kogge-Stone scan of the zero-state end states e_s held in
// carry (log2 of the segment count in steps rather than one serial pass per line):
//   forward   S_s = e_s + M S_{s-1}, s = 1 .. last-1; S_0 = e_0 is already true (the edge state)
//   backward  S_s = e_s + M S_{s+1}, s = last-1 .. 0; S_last = e_last is already true
// Step p adds M^(2^p) times the carry 2^p segments away. The segments whose maps are composed are full
// length, so M is the same for each. Every thread of the block runs the loop (it has barriers).
__device__ void carry_scan(double* carry, int nt, int cstep, int seg, int last, const IirChannel& ch, bool active,
                           bool forward) {
    // component i of thread t's carry at carry[i * nt + t]; the neighbouring segment's is cstep away
    double* cs = carry + threadIdx.x;
    for (int p = 0, k = 1; k <= last; ++p, k <<= 1) {
        const int src = forward ? seg - k : seg + k;
        const bool upd = active && (forward ? (src >= 0 && seg <= last - 1) : src <= last);
        double n0 = 0.0, n1 = 0.0, n2 = 0.0;
        if (upd) {
            const double* ps = cs + (forward ? -k : k) * cstep;
            const double p0 = ps[0], p1 = ps[nt], p2 = ps[2 * nt];
            const double(&M)[3][3] = ch.Mp[p];
            n0 = cs[0] + (M[0][0] * p0 + M[0][1] * p1 + M[0][2] * p2);
            n1 = cs[nt] + (M[1][0] * p0 + M[1][1] * p1 + M[1][2] * p2);
            n2 = cs[2 * nt] + (M[2][0] * p0 + M[2][1] * p1 + M[2][2] * p2);
        }
        __syncthreads();
        if (upd) {
            cs[0] = n0;
            cs[nt] = n1;
            cs[2 * nt] = n2;
        }
        __syncthreads();
    }
}

// The transpose's edge term: v[e] += ((B1 + B2 + B3) v[e] + (B2 + B3) v[e + step] + B3 v[e + 2 step]) / B,
// with the samples that exist (a line shorter than three samples folds what it has)
__device__ __forceinline__ void edge_fold(const Coef& k, float* base, int e, int step, int n, bool doit) {
    if (!doit) return;
    const double v0 = base[e];
    const double v1 = n > 1 ? double(base[e + step]) : 0.0;
    const double v2 = n > 2 ? double(base[e + 2 * step]) : 0.0;
    base[e] = float(v0 + (((k.B1 + k.B2) + k.B3) * v0 + (k.B2 + k.B3) * v1 + k.B3 * v2) / k.B);
}

// One full forward + backward blur of `nlines` interleaved lines of length n held in shared memory
// (line j, element i at buf[i * pitch + j]), nseg segments per line, threads = nlines * nseg. Thread t
// handles line t / nseg, segment t % nseg when seg_major, else line t % nlines, segment t / nlines; the
// channel of line j is 3 comp + j % 3. carry: shared scratch of 3 * nlines * nseg doubles, component i of
// thread t's segment at carry[i * nlines * nseg + t].
__device__ void blur_lines(float* buf, int pitch, int nlines, int n, int nseg, const IirLaunch& q, int comp,
                           double* carry, bool seg_major) {
    const int t = threadIdx.x;
    const int line = seg_major ? t / nseg : t % nlines;
    const int seg = seg_major ? t % nseg : t / nlines;
    const int cstep = seg_major ? 1 : nlines;  // carry distance between neighbouring segments of a line
    const int L = q.seg_len;
    const int a = seg * L;
    const int b = min(n, a + L);
    const IirChannel& ch = q.ch[3 * comp + line % 3];
    const bool active = ch.active != 0 && line < nlines;
    const Coef k{ch.B, ch.B1, ch.B2, ch.B3};
    float* base = buf + line;
    const int nt = nlines * nseg;
    double* cs = carry + t;

    const bool adj = q.adjoint != 0;
    // ---- forward ----
    if (active && a < n) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (seg == 0 && !adj) s1 = s2 = s3 = double(base[0]);
        seg_forward(k, base, pitch, a, b, s1, s2, s3, false);
        cs[0] = s1;
        cs[nt] = s2;
        cs[2 * nt] = s3;
    }
    __syncthreads();
    const int nseg_used = (n + L - 1) / L;
    const int last = nseg_used - 1;
    carry_scan(carry, nt, cstep, seg, last, ch, active, true);
    if (active && a < n) {
        double s1, s2, s3;
        if (seg == 0) {
            s1 = s2 = s3 = adj ? 0.0 : double(base[0]);
        } else {
            const double* prev = cs - cstep;
            s1 = prev[0];
            s2 = prev[nt];
            s3 = prev[2 * nt];
        }
        seg_forward(k, base, pitch, a, b, s1, s2, s3, true);
    }
    __syncthreads();
    if (adj) {
        // the forward blur's anticausal pass starts from y[n..n+2] = u[n-1]: its transpose adds
        // ((B1 + B2 + B3) l[n-1] + (B2 + B3) l[n-2] + B3 l[n-3]) / B to sample n-1
        edge_fold(k, base, (n - 1) * pitch, -pitch, n, active && seg == 0);
        __syncthreads();
    }
    // ---- backward ----
    if (active && a < n) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (seg == last && !adj) s1 = s2 = s3 = double(base[(n - 1) * pitch]);
        seg_backward(k, base, pitch, a, b, s1, s2, s3, false);
        cs[0] = s1;
        cs[nt] = s2;
        cs[2 * nt] = s3;
    }
    __syncthreads();
    carry_scan(carry, nt, cstep, seg, last, ch, active, false);
    if (active && a < n) {
        double s1, s2, s3;
        if (seg == last) {
            s1 = s2 = s3 = adj ? 0.0 : double(base[(n - 1) * pitch]);
        } else {
            const double* prev = cs + cstep;
            s1 = prev[0];
            s2 = prev[nt];
            s3 = prev[2 * nt];
        }
        seg_backward(k, base, pitch, a, b, s1, s2, s3, true);
    }
    __syncthreads();
    if (adj) {
        // the forward blur's causal pass starts from w[-1..-3] = x[0]: its transpose folds into sample 0
        edge_fold(k, base, 0, pitch, n, active && seg == 0);
        __syncthreads();
    }
}

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned), and the wait for all of
// this thread's copies
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__global__ void __launch_bounds__(kRowThreads) k_iir_rows(const float* __restrict__ in, IirPlanes outs, uint32_t w,
                                                          uint32_t h, const __grid_constant__ IirMixture mix) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t y = blockIdx.x;
    if (y >= h) return;
    const int n3 = int(3 * w);
    const int n3r = (n3 + 3) & ~3;  // keeps carry 16-byte aligned
    float* work = reinterpret_cast<float*>(smem);
    double* carry = reinterpret_cast<double*>(work + n3r);
    const float* src = in + size_t(y) * n3;
    const bool vec = (n3 & 3) == 0;  // rows start on 16-byte boundaries
    for (int c = 0; c < int(mix.ncomp); ++c) {
        // each component blurs the row afresh: the source row is read again (from L2 after the first)
        if (vec) {
            for (int i = threadIdx.x; i < n3 / 4; i += blockDim.x) cp_async16(work + 4 * i, src + 4 * i);
            cp_async_wait_all();
        } else {
            for (int i = threadIdx.x; i < n3; i += blockDim.x) work[i] = src[i];
        }
        __syncthreads();
        blur_lines(work, 3, 3, int(w), kSegRows, mix.rows, c, carry, true);
        float* dst = outs.p[c] + size_t(y) * n3;
        if (vec) {
            for (int i = threadIdx.x; i < n3 / 4; i += blockDim.x)
                reinterpret_cast<float4*>(dst)[i] = reinterpret_cast<const float4*>(work)[i];
        } else {
            for (int i = threadIdx.x; i < n3; i += blockDim.x) dst[i] = work[i];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kColThreads) k_iir_cols(float* raw, IirPlanes hs, float* acc, uint32_t w, uint32_t h,
                                                          const __grid_constant__ IirMixture mix,
                                                          const __grid_constant__ IirColMaps maps) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t x0 = blockIdx.x * kColPixels;
    const int px = min(kColPixels, int(w) - int(x0));
    const int nl = 3 * px;  // valid lines in this strip
    const int n = int(h);
    // [row][kColLines], boxes * box_rows rows (each box's first row 128-byte aligned: box_rows is a
    // multiple of 8 and a row is 48 bytes), then the carries, then the strip's mbarrier
    const size_t rows_alloc = size_t(maps.box_rows) * maps.boxes;
    float* strip = reinterpret_cast<float*>(smem);
    double* carry = reinterpret_cast<double*>(strip + rows_alloc * kColLines);
    const uint32_t bar = smem_addr(carry + size_t(kColLines) * kSegCols * 3);
    const size_t pitch = 3 * size_t(w);
    const size_t off = 3 * size_t(x0);
    // a full strip of a frame whose width is a multiple of 4: every strip row is three aligned float4
    const bool vec = px == kColPixels && (w & 3u) == 0;
    constexpr int kQuads = kColLines / 4;
    bool tma = vec && maps.use_tma != 0;  // the same in every thread of the CTA
    if (tma) {
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
        }
        __syncthreads();
    }
    for (int c = 0; c < int(mix.ncomp); ++c) {
        const float* src = hs.p[c];
        if (tma) {
            if (threadIdx.x == 0) {
                fence_proxy_async();  // the previous component's reads and writes of the strip come first
                mbar_arrive_expect_tx(bar, maps.boxes * maps.box_rows * uint32_t(kColLines * sizeof(float)));
                for (uint32_t k = 0; k < maps.boxes; ++k)
                    tma_load_2d(smem_addr(strip + size_t(k) * maps.box_rows * kColLines), &maps.map[c], int(off),
                                int(k * maps.box_rows), bar);
            }
            // component c completes the barrier's phase c
            const uint32_t parity = uint32_t(c) & 1u;
            bool gave_up = false, landed = true;
            if (!mbar_wait(bar, parity, maps.wait_limit)) {
                gave_up = true;
                landed = mbar_wait(bar, parity, kWaitCycles);
            }
            const int any_gave_up = __syncthreads_or(gave_up);
            const int all_landed = __syncthreads_and(landed);
            if (threadIdx.x == 0 && any_gave_up) atomicAdd(&g_iir_gave_up, 1u);
            if (!all_landed) tma = false;  // this strip and every later one by plain copies
        }
        if (tma) {
            // the strip is in place
        } else if (vec) {
            for (int i = threadIdx.x; i < n * kQuads; i += blockDim.x) {
                const int r = i / kQuads, qd = i - r * kQuads;
                cp_async16(strip + size_t(r) * kColLines + 4 * qd, src + size_t(r) * pitch + off + 4 * qd);
            }
            cp_async_wait_all();
        } else {
            for (int i = threadIdx.x; i < n * kColLines; i += blockDim.x) {
                const int r = i / kColLines, j = i % kColLines;
                strip[i] = j < nl ? src[size_t(r) * pitch + off + j] : 0.0f;
            }
        }
        __syncthreads();
        blur_lines(strip, kColLines, kColLines, n, kSegCols, mix.cols, c, carry, false);
        const bool first = c == 0, last = c + 1 == int(mix.ncomp);
        if (mix.plain) {
            // a plain blur (one component): the blurred lines as they are
            if (vec) {
                for (int i = threadIdx.x; i < n * kQuads; i += blockDim.x) {
                    const int r = i / kQuads, qd = i - r * kQuads;
                    *reinterpret_cast<float4*>(raw + size_t(r) * pitch + off + 4 * qd) =
                        *reinterpret_cast<const float4*>(strip + size_t(r) * kColLines + 4 * qd);
                }
            } else {
                for (int i = threadIdx.x; i < n * kColLines; i += blockDim.x) {
                    const int r = i / kColLines, j = i % kColLines;
                    if (j < nl) raw[size_t(r) * pitch + off + j] = strip[i];
                }
            }
        } else if (vec) {
            for (int i = threadIdx.x; i < n * kQuads; i += blockDim.x) {
                const int r = i / kQuads, qd = i - r * kQuads;
                const size_t o = size_t(r) * pitch + off + 4 * qd;
                const float4 v = *reinterpret_cast<const float4*>(strip + size_t(r) * kColLines + 4 * qd);
                const float vv[4] = {v.x, v.y, v.z, v.w};
                float av[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (!first) {
                    const float4 p = *reinterpret_cast<const float4*>(acc + o);
                    av[0] = p.x;
                    av[1] = p.y;
                    av[2] = p.z;
                    av[3] = p.w;
                }
                float4 rw = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (last) rw = *reinterpret_cast<const float4*>(raw + o);
                float rr[4] = {rw.x, rw.y, rw.z, rw.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int ch3 = (4 * qd + e) % 3;
                    const float wc = mix.weight[c][ch3];
                    av[e] = first ? 0.0f + wc * vv[e] : av[e] + wc * vv[e];
                    if (last) rr[e] = mix.mix_a[ch3] * rr[e] + mix.mix_b[ch3] * av[e];
                }
                if (last) *reinterpret_cast<float4*>(raw + o) = make_float4(rr[0], rr[1], rr[2], rr[3]);
                else *reinterpret_cast<float4*>(acc + o) = make_float4(av[0], av[1], av[2], av[3]);
            }
        } else {
            for (int i = threadIdx.x; i < n * kColLines; i += blockDim.x) {
                const int r = i / kColLines, j = i % kColLines;
                if (j >= nl) continue;
                const size_t o = size_t(r) * pitch + off + j;
                const float v = strip[i];
                const float wc = mix.weight[c][j % 3];
                const float a = first ? 0.0f + wc * v : acc[o] + wc * v;
                if (last) {
                    const float m0 = mix.mix_a[j % 3], m1 = mix.mix_b[j % 3];
                    raw[o] = m0 * raw[o] + m1 * a;
                } else {
                    acc[o] = a;
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace

size_t iir_rows_smem(uint32_t w) {
    const size_t n3r = (3 * size_t(w) + 3) & ~size_t(3);
    return n3r * sizeof(float) + size_t(3) * kSegRows * 3 * sizeof(double);
}

namespace {
// The strip's boxes: ceil(h / 256) of them, each a multiple of 8 rows (at most 256) and together at least h.
struct ColBoxes {
    uint32_t rows, boxes;
};
ColBoxes col_boxes(uint32_t h) {
    const uint32_t boxes = h > 0 ? (h + 255u) / 256u : 1u;
    const uint32_t per = (h + boxes - 1u) / boxes;
    return {(per + 7u) & ~7u, boxes};
}
}  // namespace

size_t iir_cols_smem(uint32_t h) {
    const ColBoxes cb = col_boxes(h);
    return size_t(cb.rows) * cb.boxes * kColLines * sizeof(float) + size_t(kColLines) * kSegCols * 3 * sizeof(double) +
           sizeof(uint64_t);
}

// The column segment length: at least n / nseg, and with nlines L = nlines (mod 32), so that a warp's
// lanes (line t % nlines, segment t / nlines, sample i) address floats equal to t + nlines i modulo 32
// and never share a shared-memory bank (L = 1 (mod 8) for twelve lines).
namespace {
int seg_len(uint32_t n, int nseg, int nlines) {
    int g = 32;
    while (nlines % g != 0) g /= 2;  // gcd(nlines, 32)
    const int m = 32 / g;
    const int L0 = int((n + uint32_t(nseg) - 1) / uint32_t(nseg));
    return L0 + ((1 - L0) % m + m) % m;
}
}  // namespace

// rows run segment-major (a warp's lanes: one line, 32 consecutive segments, addresses 3 L t + const):
// any odd L keeps them in distinct banks
int iir_row_seg_len(uint32_t w) {
    const int L0 = int((w + uint32_t(kSegRows) - 1) / uint32_t(kSegRows));
    return L0 | 1;
}
int iir_col_seg_len(uint32_t h) { return seg_len(h, kSegCols, kColLines); }

bool iir_mixture_fits(uint32_t w, uint32_t h) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return iir_rows_smem(w) <= size_t(optin) && iir_cols_smem(h) <= size_t(optin);
}

namespace {
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, looked up once (null when the driver cannot give it)
EncodeTiled encode_tiled() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(f);
    });
    return fn;
}

std::atomic<long long> g_wait_limit{0};  // set_iir_wait_limit: 0 the full limit

// The tensor maps of the column pass's component planes: each a 2-D tensor of 3 w floats x h rows (row
// pitch 12 w bytes), read in 12 x box_rows boxes. False (plain copies) for a width that is not a multiple
// of 4 (the rows and the strips' x coordinates would leave 16-byte alignment), a plane not on a 16-byte
// boundary, or a map the driver refuses.
bool col_maps(IirColMaps& maps, const IirPlanes& planes, uint32_t ncomp, uint32_t w, uint32_t h) {
    const ColBoxes cb = col_boxes(h);
    maps.box_rows = cb.rows;
    maps.boxes = cb.boxes;
    const long long lim = g_wait_limit.load();
    maps.wait_limit = lim > 0 ? lim : kWaitCycles;
    maps.use_tma = 0;
    const EncodeTiled enc = encode_tiled();
    if (!kColTma || !enc || (w & 3u) != 0u) return false;
    const cuuint64_t dims[2] = {cuuint64_t(3) * w, h};
    const cuuint64_t strides[1] = {cuuint64_t(3) * w * sizeof(float)};
    const cuuint32_t box[2] = {cuuint32_t(kColLines), cb.rows};
    const cuuint32_t estr[2] = {1, 1};
    for (uint32_t c = 0; c < ncomp; ++c) {
        if ((reinterpret_cast<uintptr_t>(planes.p[c]) & 15u) != 0u) return false;
        if (enc(&maps.map[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, planes.p[c], dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    maps.use_tma = 1;
    return true;
}
}  // namespace

void set_iir_wait_limit(long long cycles) { g_wait_limit.store(cycles); }

uint32_t take_iir_waits_given_up(cudaStream_t s) {
    unsigned int v = 0, zero = 0;
    cudaMemcpyFromSymbolAsync(&v, g_iir_gave_up, sizeof(v), 0, cudaMemcpyDeviceToHost, s);
    cudaMemcpyToSymbolAsync(g_iir_gave_up, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    return v;
}

void iir_mixture(const float* src, float* raw, float* const* tmp, float* acc, uint32_t w, uint32_t h,
                 const IirMixture& m, cudaStream_t s) {
    IirPlanes planes{};
    for (uint32_t c = 0; c < m.ncomp; ++c) planes.p[c] = tmp[c];
    const size_t sr = iir_rows_smem(w), sc = iir_cols_smem(h);
    ensure_smem(reinterpret_cast<const void*>(k_iir_rows), int(sr));
    ensure_smem(reinterpret_cast<const void*>(k_iir_cols), int(sc));
    IirColMaps maps{};
    col_maps(maps, planes, m.ncomp, w, h);
    {
        Probe p("iir_rows", s);
        k_iir_rows<<<h, kRowThreads, sr, s>>>(src, planes, w, h, m);
    }
    {
        Probe p("iir_cols", s);
        k_iir_cols<<<(w + kColPixels - 1) / kColPixels, kColThreads, sc, s>>>(raw, planes, acc, w, h, m, maps);
    }
}

}  // namespace spkb::dev
