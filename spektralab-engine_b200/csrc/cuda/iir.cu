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
//      entry state through L steps of the homogeneous recurrence (a short serial pass per line);
//   3. every segment recomputes from its true entry state and stores its values.
// State and the carries are binary64 (the reference keeps double-float state on its GPU and double
// state on its host copy); x, u and y are stored as binary32 exactly as there.
//
// k_iir_rows: one CTA per image row; the row (3 w floats) in shared memory; every mixture component
//             blurred in turn from the same row and written to its own plane.
// k_iir_cols: one CTA per strip of 4 pixel columns (12 lines); every component's row result blurred
//             down the columns in turn; the mixture accumulated as the reference's fused passes do
//             (acc = 0 + w0 y0, acc = acc + w_k y_k) and the halation mix raw := a raw + b acc written
//             in place of raw.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "iir.hpp"

namespace spkb::dev {

namespace {

constexpr int kSegRows = 64;       // segments per channel line in a row
constexpr int kRowThreads = 3 * kSegRows;
constexpr int kColPixels = 4;       // pixels per column strip
constexpr int kColLines = 3 * kColPixels;
constexpr int kSegCols = 32;        // segments per column line (two 4K strips per SM)
constexpr int kColThreads = kColLines * kSegCols;

struct Coef {
    double B, B1, B2, B3;
};

__device__ __forceinline__ double step(const Coef& k, double x, double s1, double s2, double s3) {
    // the product with the newest state last, so that only one multiply-add waits on it
    return fma(k.B1, s1, fma(k.B3, s3, fma(k.B2, s2, k.B * x)));
}

// Forward pass over one segment [a, b) of a line in shared memory (element i at base[i * stride]).
// Zero-state run: returns the end state. Writing run: from `in` state, stores float(w) back.
__device__ __forceinline__ void seg_forward(const Coef& k, float* base, int stride, int a, int b, double& s1,
                                            double& s2, double& s3, bool write) {
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
    for (int i = b - 1; i >= a; --i) {
        const double t = step(k, double(base[i * stride]), s1, s2, s3);
        s3 = s2;
        s2 = s1;
        s1 = t;
        if (write) base[i * stride] = float(t);
    }
}

// One full forward + backward blur of `nlines` interleaved lines of length n held in shared memory
// (line j, element i at buf[i * pitch + j]); nseg segments per line; threads = nlines * nseg, thread
// t handles line t % nlines, segment t / nlines. carry: shared scratch of nlines * nseg * 3 doubles.
__device__ void blur_lines(float* buf, int pitch, int nlines, int n, int nseg, const IirLaunch& q, const int* comp_line,
                           double* carry) {
    const int t = threadIdx.x;
    const int line = t % nlines;
    const int seg = t / nlines;
    const int L = q.seg_len;
    const int a = seg * L;
    const int b = min(n, a + L);
    const IirChannel& ch = q.ch[comp_line[line]];
    const bool active = ch.active != 0;
    const Coef k{ch.B, ch.B1, ch.B2, ch.B3};
    float* base = buf + line;
    double* cs = carry + (size_t(seg) * nlines + line) * 3;

    // ---- forward ----
    if (active && a < n) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (seg == 0) s1 = s2 = s3 = double(base[0]);
        seg_forward(k, base, pitch, a, b, s1, s2, s3, false);
        cs[0] = s1;
        cs[1] = s2;
        cs[2] = s3;
    }
    __syncthreads();
    const int nseg_used = (n + L - 1) / L;
    const int last = nseg_used - 1;
    if (active && seg == 0) {  // serial carry: true end state of every segment that has a successor
        for (int s = 1; s < last; ++s) {  // segments 1 .. last-1 are full length L
            const double* prev = carry + (size_t(s - 1) * nlines + line) * 3;
            double* cur = carry + (size_t(s) * nlines + line) * 3;
            const double p0 = prev[0], p1 = prev[1], p2 = prev[2];
            cur[0] = cur[0] + (ch.M[0][0] * p0 + ch.M[0][1] * p1 + ch.M[0][2] * p2);
            cur[1] = cur[1] + (ch.M[1][0] * p0 + ch.M[1][1] * p1 + ch.M[1][2] * p2);
            cur[2] = cur[2] + (ch.M[2][0] * p0 + ch.M[2][1] * p1 + ch.M[2][2] * p2);
        }
    }
    __syncthreads();
    if (active && a < n) {
        double s1, s2, s3;
        if (seg == 0) {
            s1 = s2 = s3 = double(base[0]);
        } else {
            const double* prev = carry + (size_t(seg - 1) * nlines + line) * 3;
            s1 = prev[0];
            s2 = prev[1];
            s3 = prev[2];
        }
        seg_forward(k, base, pitch, a, b, s1, s2, s3, true);
    }
    __syncthreads();
    // ---- backward ----
    if (active && a < n) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (seg == last) s1 = s2 = s3 = double(base[(n - 1) * pitch]);
        seg_backward(k, base, pitch, a, b, s1, s2, s3, false);
        cs[0] = s1;
        cs[1] = s2;
        cs[2] = s3;
    }
    __syncthreads();
    if (active && seg == 0) {  // serial carry from the right end leftwards; full segments only
        for (int s = last - 1; s >= 0; --s) {
            const double* prev = carry + (size_t(s + 1) * nlines + line) * 3;
            double* cur = carry + (size_t(s) * nlines + line) * 3;
            const double p0 = prev[0], p1 = prev[1], p2 = prev[2];
            cur[0] = cur[0] + (ch.M[0][0] * p0 + ch.M[0][1] * p1 + ch.M[0][2] * p2);
            cur[1] = cur[1] + (ch.M[1][0] * p0 + ch.M[1][1] * p1 + ch.M[1][2] * p2);
            cur[2] = cur[2] + (ch.M[2][0] * p0 + ch.M[2][1] * p1 + ch.M[2][2] * p2);
        }
    }
    __syncthreads();
    if (active && a < n) {
        double s1, s2, s3;
        if (seg == last) {
            s1 = s2 = s3 = double(base[(n - 1) * pitch]);
        } else {
            const double* prev = carry + (size_t(seg + 1) * nlines + line) * 3;
            s1 = prev[0];
            s2 = prev[1];
            s3 = prev[2];
        }
        seg_backward(k, base, pitch, a, b, s1, s2, s3, true);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kRowThreads) k_iir_rows(const float* __restrict__ in, IirPlanes outs, uint32_t w,
                                                          uint32_t h, const __grid_constant__ IirMixture mix) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t y = blockIdx.x;
    if (y >= h) return;
    const int n3 = int(3 * w);
    const int n3r = (n3 + 3) & ~3;  // keeps work and carry 16-byte aligned
    float* row = reinterpret_cast<float*>(smem);
    float* work = row + n3r;
    double* carry = reinterpret_cast<double*>(work + n3r);
    const float* src = in + size_t(y) * n3;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) row[i] = src[i];
    __syncthreads();
    for (int c = 0; c < int(mix.ncomp); ++c) {
        for (int i = threadIdx.x; i < n3; i += blockDim.x) work[i] = row[i];
        __syncthreads();
        const int comp_line[3] = {3 * c + 0, 3 * c + 1, 3 * c + 2};
        blur_lines(work, 3, 3, int(w), kSegRows, mix.rows, comp_line, carry);
        float* dst = outs.p[c] + size_t(y) * n3;
        for (int i = threadIdx.x; i < n3; i += blockDim.x) dst[i] = work[i];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kColThreads) k_iir_cols(float* raw, IirPlanes hs, float* acc, uint32_t w, uint32_t h,
                                                          const __grid_constant__ IirMixture mix) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t x0 = blockIdx.x * kColPixels;
    const int px = min(kColPixels, int(w) - int(x0));
    const int nl = 3 * px;  // valid lines in this strip
    const int n = int(h);
    float* strip = reinterpret_cast<float*>(smem);  // [row][kColLines]
    double* carry = reinterpret_cast<double*>(strip + size_t(n) * kColLines);
    const size_t pitch = 3 * size_t(w);
    const size_t off = 3 * size_t(x0);
    for (int c = 0; c < int(mix.ncomp); ++c) {
        const float* src = hs.p[c];
        for (int i = threadIdx.x; i < n * kColLines; i += blockDim.x) {
            const int r = i / kColLines, j = i % kColLines;
            strip[i] = j < nl ? src[size_t(r) * pitch + off + j] : 0.0f;
        }
        __syncthreads();
        int comp_line[kColLines];
#pragma unroll
        for (int j = 0; j < kColLines; ++j) comp_line[j] = 3 * c + j % 3;
        blur_lines(strip, kColLines, kColLines, n, kSegCols, mix.cols, comp_line, carry);
        const float wgt[3] = {mix.weight[c][0], mix.weight[c][1], mix.weight[c][2]};
        const bool last = c + 1 == int(mix.ncomp);
        for (int i = threadIdx.x; i < n * kColLines; i += blockDim.x) {
            const int r = i / kColLines, j = i % kColLines;
            if (j >= nl) continue;
            const size_t o = size_t(r) * pitch + off + j;
            const float v = strip[i];
            const float wc = wgt[j % 3];
            const float a = c == 0 ? 0.0f + wc * v : acc[o] + wc * v;
            if (last) {
                const float m0 = mix.mix_a[j % 3], m1 = mix.mix_b[j % 3];
                raw[o] = m0 * raw[o] + m1 * a;
            } else {
                acc[o] = a;
            }
        }
        __syncthreads();
    }
}

}  // namespace

size_t iir_rows_smem(uint32_t w) {
    const size_t n3r = (3 * size_t(w) + 3) & ~size_t(3);
    return 2 * n3r * sizeof(float) + size_t(3) * kSegRows * 3 * sizeof(double);
}

size_t iir_cols_smem(uint32_t h) {
    return size_t(h) * kColLines * sizeof(float) + size_t(kColLines) * kSegCols * 3 * sizeof(double);
}

int iir_row_segments() { return kSegRows; }
int iir_col_segments() { return kSegCols; }

bool iir_mixture_fits(uint32_t w, uint32_t h) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return iir_rows_smem(w) <= size_t(optin) && iir_cols_smem(h) <= size_t(optin);
}

void iir_mixture(float* raw, float* const* tmp, float* acc, uint32_t w, uint32_t h, const IirMixture& m,
                 cudaStream_t s) {
    IirPlanes planes{};
    for (uint32_t c = 0; c < m.ncomp; ++c) planes.p[c] = tmp[c];
    const size_t sr = iir_rows_smem(w), sc = iir_cols_smem(h);
    cudaFuncSetAttribute(k_iir_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sr));
    cudaFuncSetAttribute(k_iir_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sc));
    {
        Probe p("iir_rows", s);
        k_iir_rows<<<h, kRowThreads, sr, s>>>(raw, planes, w, h, m);
    }
    {
        Probe p("iir_cols", s);
        k_iir_cols<<<(w + kColPixels - 1) / kColPixels, kColThreads, sc, s>>>(raw, planes, acc, w, h, m);
    }
}

}  // namespace spkb::dev
