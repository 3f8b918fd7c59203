// The scanner stage in one pass: lens blur (FIR), unsharp mask (FIR + combine), output matrix, transfer
// function and RGBA16 encode, over 32 x 32 pixel tiles staged in shared memory.
//
// Reference: src/fx/scanner.cpp:16-31 (blur, then (1 + a) x - a G(x)), kernels/fx_blur.metal:20-78
// (FIR: taps -r..r ascending, binary32 accumulator from 0, half-sample symmetric reflection at the
// edges, a vertical pass then a horizontal pass) and kernels/print.metal:350-366 (encode).
//
// Every intermediate value is the one the separate passes compute: each pass is evaluated only at
// pixels inside the image, in the same tap order, and where a pass reads past an edge it reads the
// value at the reflected pixel. The vertical passes do not mix columns, so a column loaded from the
// reflected source column already carries the reflected result; after the lens blur's horizontal pass
// the tile copies the reflected values into the (at most r2 wide) border that the unsharp pass reads.
//
// Shared memory (floats, interleaved RGB rows), R = r1 + r2:
//   A: the print output with an R halo (TH + 2R rows x 3 (TW + 2R)), later the lens-blurred tile with an
//      r2 halo (TH + 2 r2 rows x 3 (TW + 2 r2))
//   B: the lens blur's vertical pass (TH + 2 r2 rows x 3 (TW + 2R)), later the unsharp vertical pass
//      (TH rows x 3 (TW + 2 r2))
#include <cuda_runtime.h>
#include <stdint.h>

#include "../kernel_args.h"
#include "encode.cuh"
#include "launch.hpp"

namespace spkb::dev {

namespace {

// threads per tile CTA (4K scanner: 0.326 ms at 128, 0.209 at 256, 0.191 at 512; the pixels are the same)
#ifndef SPKB_SCAN_THREADS
#define SPKB_SCAN_THREADS 512
#endif
constexpr int kTW = 32, kTH = 32, kThreads = SPKB_SCAN_THREADS, kWarps = kThreads / 32;
static_assert(uint32_t(kTH) == scan_tile_rows(), "row bands start on tile rows");

// half-sample symmetric reflection, exact for p in [-n, 2n)
__device__ __forceinline__ int reflect_near(int p, int n) { return p < 0 ? -1 - p : (p >= n ? 2 * n - 1 - p : p); }

// One 32 x 32 output tile at (x0, y0) of a frame; smem as sized by scan_smem_bytes for the radii.
template <int R1, int R2>
__device__ __forceinline__ void scan_tile(const ScanArgs& a, const float* __restrict__ rgb, uint16_t* __restrict__ out,
                                          int w, int h, int x0, int y0, float* smem) {
    const int r1 = R1 >= 0 ? R1 : a.r1, r2 = R2 >= 0 ? R2 : a.r2, R = r1 + r2;
    const int PC = 3 * (kTW + 2 * R);  // floats per row of the print tile and the first vertical pass
    const int PR = kTH + 2 * R;
    const int BR = kTH + 2 * r2;       // rows of the lens-blurred tile
    const int BC = 3 * (kTW + 2 * r2);
    float* A = smem;
    float* B = smem + PR * PC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // 1. the print output at (y0 - R + i, x0 - R + j), reflected; pixels more than R past an edge are
    //    never read and load a clamped pixel. A tile whose haloed columns lie inside the frame reads each
    //    row's floats contiguously, with no per-element reflection.
    const bool inner_x = x0 - R >= 0 && x0 + kTW + R <= w;
    for (int i = warp; i < PR; i += kWarps) {
        const int yy = min(max(reflect_near(y0 - R + i, h), 0), h - 1);
        const float* row = rgb + size_t(yy) * size_t(w) * 3;
        if (inner_x) {
            const float* seg = row + 3 * (x0 - R);
            for (int f = lane; f < PC; f += 32) A[i * PC + f] = __ldg(seg + f);
            continue;
        }
        for (int f = lane; f < PC; f += 32) {
            const int j = f / 3, c = f - 3 * j;
            const int xx = min(max(reflect_near(x0 - R + j, w), 0), w - 1);
            A[i * PC + f] = __ldg(row + 3 * xx + c);
        }
    }
    __syncthreads();

    if constexpr (R1 >= 0 && R2 >= 0) {
        // 2. lens blur, vertical, with register windows: a thread takes kVRows consecutive output rows of
        //    one column and reads each input row once; every output is still sum_k t1[k] A[i + k] from 0,
        //    k ascending
        constexpr int T1 = 2 * R1 + 1, PCc = 3 * (kTW + 2 * (R1 + R2)), PRc = kTH + 2 * (R1 + R2);
        constexpr int BRc = kTH + 2 * R2, BCc = 3 * (kTW + 2 * R2);
        constexpr int kVRows = 6, NB = (BRc + kVRows - 1) / kVRows;
        for (int item = threadIdx.x; item < PCc * NB; item += kThreads) {
            const int f = item % PCc, i0 = (item / PCc) * kVRows;
            float acc[kVRows];
#pragma unroll
            for (int o = 0; o < kVRows; ++o) acc[o] = 0.0f;
#pragma unroll
            for (int j = 0; j < kVRows + T1 - 1; ++j) {
                if (i0 + j < PRc) {
                    const float v = A[(i0 + j) * PCc + f];
#pragma unroll
                    for (int o = 0; o < kVRows; ++o)
                        if (j - o >= 0 && j - o < T1) acc[o] += a.t1[j - o] * v;
                }
            }
#pragma unroll
            for (int o = 0; o < kVRows; ++o) {
                const int i = i0 + o, yy = y0 - R2 + i;
                if (i < BRc && yy >= 0 && yy < h) B[i * PCc + f] = acc[o];
            }
        }
        __syncthreads();

        // 3. lens blur, horizontal, with register windows: a thread takes kHPix consecutive output pixels
        //    of one channel in one row
        constexpr int kHPix = 4, NG = (kTW + 2 * R2 + kHPix - 1) / kHPix;
        for (int item = threadIdx.x; item < BRc * 3 * NG; item += kThreads) {
            const int i = item / (3 * NG), rem = item - i * (3 * NG), c = rem % 3, j0 = (rem / 3) * kHPix;
            const int yy = y0 - R2 + i;
            if (yy < 0 || yy >= h) continue;
            float acc[kHPix];
#pragma unroll
            for (int o = 0; o < kHPix; ++o) acc[o] = 0.0f;
            const float* brow = B + i * PCc + c;
#pragma unroll
            for (int q = 0; q < kHPix + T1 - 1; ++q) {
                if (j0 + q < kTW + 2 * (R1 + R2)) {
                    const float v = brow[3 * (j0 + q)];
#pragma unroll
                    for (int o = 0; o < kHPix; ++o)
                        if (q - o >= 0 && q - o < T1) acc[o] += a.t1[q - o] * v;
                }
            }
#pragma unroll
            for (int o = 0; o < kHPix; ++o) {
                const int jb = j0 + o;
                if (jb >= kTW + 2 * R2) break;
                if (!inner_x) {
                    const int xx = x0 - R2 + jb;
                    if (xx < 0 || xx >= w) continue;
                }
                A[i * BCc + 3 * jb + c] = acc[o];
            }
        }
        __syncthreads();
    } else {
    // 2. lens blur, vertical: rows y0 - r2 + i inside the image, every column of the tile
    for (int i = warp; i < BR; i += kWarps) {
        const int yy = y0 - r2 + i;
        if (yy < 0 || yy >= h) continue;
        for (int f = lane; f < PC; f += 32) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * r1; ++k) acc += a.t1[k] * A[(i + k) * PC + f];
            B[i * PC + f] = acc;
        }
    }
    __syncthreads();

    // 3. lens blur, horizontal: pixels (y0 - r2 + i, x0 - r2 + jb) inside the image, into A
    for (int i = warp; i < BR; i += kWarps) {
        const int yy = y0 - r2 + i;
        if (yy < 0 || yy >= h) continue;
        for (int fb = lane; fb < BC; fb += 32) {
            if (!inner_x) {
                const int xx = x0 - r2 + fb / 3;
                if (xx < 0 || xx >= w) continue;
            }
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * r1; ++k) acc += a.t1[k] * B[i * PC + fb + 3 * k];
            A[i * BC + fb] = acc;
        }
    }
    __syncthreads();
    }

    if (r2 > 0) {
        // 4. the border up to r2 past an edge takes the lens-blurred value of the reflected pixel
        if (x0 - r2 < 0 || x0 + kTW + r2 > w || y0 - r2 < 0 || y0 + kTH + r2 > h) {
            for (int i = warp; i < BR; i += kWarps) {
                const int yy = y0 - r2 + i;
                if (yy < -r2 || yy >= h + r2) continue;
                const bool row_out = yy < 0 || yy >= h;
                const int is = reflect_near(yy, h) - (y0 - r2);
                for (int fb = lane; fb < BC; fb += 32) {
                    const int jb = fb / 3, c = fb - 3 * jb;
                    const int xx = x0 - r2 + jb;
                    if (xx < -r2 || xx >= w + r2) continue;
                    if (!row_out && xx >= 0 && xx < w) continue;
                    const int js = reflect_near(xx, w) - (x0 - r2);
                    A[i * BC + fb] = A[is * BC + 3 * js + c];
                }
            }
            __syncthreads();
        }
        // 5. unsharp blur, vertical: the tile's rows inside the image, every column of the blurred tile
        if constexpr (R2 >= 0) {
            // register windows of kURows rows per thread, as in step 2
            constexpr int T2 = 2 * R2 + 1, BCc = 3 * (kTW + 2 * R2), BRc = kTH + 2 * R2;
            constexpr int kURows = 8, NU = kTH / kURows;
            for (int item = threadIdx.x; item < BCc * NU; item += kThreads) {
                const int fb = item % BCc, i0 = (item / BCc) * kURows;
                float acc[kURows];
#pragma unroll
                for (int o = 0; o < kURows; ++o) acc[o] = 0.0f;
#pragma unroll
                for (int j = 0; j < kURows + T2 - 1; ++j) {
                    if (i0 + j < BRc) {
                        const float v = A[(i0 + j) * BCc + fb];
#pragma unroll
                        for (int o = 0; o < kURows; ++o)
                            if (j - o >= 0 && j - o < T2) acc[o] += a.t2[j - o] * v;
                    }
                }
#pragma unroll
                for (int o = 0; o < kURows; ++o)
                    if (y0 + i0 + o < h) B[(i0 + o) * BCc + fb] = acc[o];
            }
        } else {
        for (int i = warp; i < kTH; i += kWarps) {
            if (y0 + i >= h) break;
            for (int fb = lane; fb < BC; fb += 32) {
                float acc = 0.0f;
#pragma unroll
                for (int k = 0; k <= 2 * r2; ++k) acc += a.t2[k] * A[(i + k) * BC + fb];
                B[i * BC + fb] = acc;
            }
        }
        }
        __syncthreads();
    }

    // 6. unsharp horizontal pass and combine, matrix, transfer function, RGBA16: a pixel per lane
    const EncodeArgs& e = a.e;
    for (int i = warp; i < kTH; i += kWarps) {
        const int yy = y0 + i, xx = x0 + lane;
        if (yy >= h) break;
        if (xx >= w) continue;
        const float* bc = A + (i + r2) * BC + 3 * (lane + r2);
        float v0 = bc[0], v1 = bc[1], v2 = bc[2];
        if (e.unsharp) {
            const float* vr = B + i * BC + 3 * lane;
            float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * r2; ++k) {
                g0 += a.t2[k] * vr[3 * k];
                g1 += a.t2[k] * vr[3 * k + 1];
                g2 += a.t2[k] * vr[3 * k + 2];
            }
            v0 = e.lincomb_a * v0 + e.lincomb_b * g0;
            v1 = e.lincomb_a * v1 + e.lincomb_b * g1;
            v2 = e.lincomb_a * v2 + e.lincomb_b * g2;
        }
        edr_tone(e, v0, v1, v2);
        if (e.cctf_active) {
            float m0, m1, m2;
            mat_apply(e.m_nid, v0, v1, v2, m0, m1, m2);
            v0 = cctf_encode(m0, e.cctf_mode);
            v1 = cctf_encode(m1, e.cctf_mode);
            v2 = cctf_encode(m2, e.cctf_mode);
        }
        ushort4 p;
        p.x = encode16(v0);
        p.y = encode16(v1);
        p.z = encode16(v2);
        p.w = 65535;
        reinterpret_cast<ushort4*>(out)[size_t(yy) * e.stride + xx] = p;
    }
}

template <int R1, int R2>
__global__ void __launch_bounds__(kThreads) k_scan_encode(const float* __restrict__ rgb, uint16_t* __restrict__ out,
                                                          int w, int h, int row0, const __grid_constant__ ScanArgs a) {
    extern __shared__ float smem[];
    scan_tile<R1, R2>(a, rgb, out, w, h, blockIdx.x * kTW, row0 + int(blockIdx.y) * kTH, smem);
}

// The scanner stage of many frames in one persistent launch: the CTAs take tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... of the frames' concatenated tile lists (row-major within a frame).
template <int R1, int R2>
__global__ void __launch_bounds__(kThreads) k_scan_encode_batch(const BatchScanFrame* __restrict__ frames,
                                                                uint32_t n_frames, uint32_t n_tiles) {
    extern __shared__ float smem[];
    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        uint32_t lo = 0, hi = n_frames;  // the last frame whose first tile is <= t
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (frames[mid].first_tile <= t) lo = mid;
            else hi = mid;
        }
        const BatchScanFrame& f = frames[lo];
        const uint32_t local = t - f.first_tile;
        const uint32_t ty = local / f.tiles_x, tx = local - ty * f.tiles_x;
        __syncthreads();  // the previous tile's reads of shared memory are done
        scan_tile<R1, R2>(f.args, f.rgb, f.out, int(f.w), int(f.h), int(tx) * kTW, int(ty) * kTH, smem);
    }
}

// A separable FIR Gaussian with one tap vector for the three channels, both passes in one tiled kernel:
// the vertical pass at the tile's rows (every column of the haloed tile; a halo column holds the
// reflected source column, so its vertical result is that of the reflected column), then the horizontal
// pass. out must not alias in (neighbouring tiles read in's halo).
template <int R>
__global__ void __launch_bounds__(kThreads) k_fir_tile(const float* __restrict__ in, float* __restrict__ out, int w,
                                                       int h, const __grid_constant__ ScanArgs a) {
    extern __shared__ float smem[];
    const int r = R >= 0 ? R : a.r1;
    const int PC = 3 * (kTW + 2 * r), PR = kTH + 2 * r;
    float* A = smem;
    float* B = smem + PR * PC;
    const int x0 = blockIdx.x * kTW, y0 = blockIdx.y * kTH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool inner_x = x0 - r >= 0 && x0 + kTW + r <= w;  // the haloed columns lie inside the frame
    for (int i = warp; i < PR; i += kWarps) {
        const int yy = min(max(reflect_near(y0 - r + i, h), 0), h - 1);
        const float* row = in + size_t(yy) * size_t(w) * 3;
        if (inner_x) {
            const float* seg = row + 3 * (x0 - r);
            for (int f = lane; f < PC; f += 32) A[i * PC + f] = __ldg(seg + f);
            continue;
        }
        for (int f = lane; f < PC; f += 32) {
            const int j = f / 3, c = f - 3 * j;
            const int xx = min(max(reflect_near(x0 - r + j, w), 0), w - 1);
            A[i * PC + f] = __ldg(row + 3 * xx + c);
        }
    }
    __syncthreads();
    if constexpr (R >= 0) {
        // register windows: a thread takes kFRows consecutive rows of one column and reads each input row
        // once; every output is still sum_k t[k] A[i + k] from 0, k ascending
        constexpr int T = 2 * R + 1, PCc = 3 * (kTW + 2 * R), kFRows = 8, NB = kTH / kFRows;
        for (int item = threadIdx.x; item < PCc * NB; item += kThreads) {
            const int f = item % PCc, i0 = (item / PCc) * kFRows;
            float acc[kFRows];
#pragma unroll
            for (int o = 0; o < kFRows; ++o) acc[o] = 0.0f;
#pragma unroll
            for (int j = 0; j < kFRows + T - 1; ++j) {
                const float v = A[(i0 + j) * PCc + f];
#pragma unroll
                for (int o = 0; o < kFRows; ++o)
                    if (j - o >= 0 && j - o < T) acc[o] += a.t1[j - o] * v;
            }
#pragma unroll
            for (int o = 0; o < kFRows; ++o)
                if (y0 + i0 + o < h) B[(i0 + o) * PCc + f] = acc[o];
        }
    } else {
    for (int i = warp; i < kTH; i += kWarps) {
        if (y0 + i >= h) break;
        for (int f = lane; f < PC; f += 32) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * r; ++k) acc += a.t1[k] * A[(i + k) * PC + f];
            B[i * PC + f] = acc;
        }
    }
    }
    __syncthreads();
    const int OC = 3 * kTW;
    for (int i = warp; i < kTH; i += kWarps) {
        const int yy = y0 + i;
        if (yy >= h) break;
        float* orow = out + size_t(yy) * size_t(w) * 3 + size_t(x0) * 3;
        const int lim = 3 * min(kTW, w - x0);
        for (int f = lane; f < OC; f += 32) {
            if (f >= lim) break;
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k <= 2 * r; ++k) acc += a.t1[k] * B[i * PC + f + 3 * k];
            orow[f] = acc;
        }
    }
}

size_t scan_smem_bytes(int r1, int r2) {
    const int R = r1 + r2;
    return size_t((kTH + 2 * R) + (kTH + 2 * r2)) * size_t(3 * (kTW + 2 * R)) * sizeof(float);
}

template <int R1, int R2>
void launch_scan(const float* rgb, uint16_t* out, uint32_t w, uint32_t h, uint32_t row0, uint32_t row1,
                 const ScanArgs& a, cudaStream_t s) {
    const size_t smem = scan_smem_bytes(a.r1, a.r2);  // at most 96 KB (r1 = r2 = 9)
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode<R1, R2>), int(smem));
    const dim3 g((w + kTW - 1) / kTW, (row1 - row0 + kTH - 1) / kTH);
    k_scan_encode<R1, R2><<<g, kThreads, smem, s>>>(rgb, out, int(w), int(h), int(row0), a);
}

}  // namespace

bool scan_encode_fits(uint32_t w, uint32_t h, int r1, int r2) {
    const int R = r1 + r2;
    return r1 >= 0 && r2 >= 0 && r1 <= SPKB_FIR_MAX_R && r2 <= SPKB_FIR_MAX_R && w >= uint32_t(R) + 1 &&
           h >= uint32_t(R) + 1 && (uint64_t(h) + kTH - 1) / kTH <= 65535u;
}

void scan_encode_rows(const float* rgb, uint16_t* out, uint32_t w, uint32_t h, uint32_t row0, uint32_t row1,
                      const ScanArgs& a, cudaStream_t s) {
    if (uint64_t(w) * h == 0 || row1 <= row0) return;
    Probe p("scan_encode", s);
    if (a.r1 == 5 && a.r2 == 2) launch_scan<5, 2>(rgb, out, w, h, row0, row1, a, s);
    else if (a.r1 == 0 && a.r2 == 2) launch_scan<0, 2>(rgb, out, w, h, row0, row1, a, s);
    else launch_scan<-1, -1>(rgb, out, w, h, row0, row1, a, s);
}

void scan_encode(const float* rgb, uint16_t* out, uint32_t w, uint32_t h, const ScanArgs& a, cudaStream_t s) {
    scan_encode_rows(rgb, out, w, h, 0, h, a, s);
}

namespace {
template <int R1, int R2>
void launch_scan_batch(const BatchScanFrame* frames, uint32_t n_frames, uint32_t n_tiles, uint32_t ctas, size_t smem,
                       cudaStream_t s) {
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode_batch<R1, R2>), int(smem));
    k_scan_encode_batch<R1, R2><<<ctas, kThreads, smem, s>>>(frames, n_frames, n_tiles);
}
}  // namespace

void scan_prepare() {
    const int max_smem = int(scan_smem_bytes(SPKB_FIR_MAX_R, SPKB_FIR_MAX_R));
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode<5, 2>), int(scan_smem_bytes(5, 2)));
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode<0, 2>), int(scan_smem_bytes(0, 2)));
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode<-1, -1>), max_smem);
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode_batch<5, 2>), int(scan_smem_bytes(5, 2)));
    ensure_smem(reinterpret_cast<const void*>(k_scan_encode_batch<-1, -1>), max_smem);
}

uint32_t scan_tiles(uint32_t w, uint32_t h) { return ((w + kTW - 1) / kTW) * ((h + kTH - 1) / kTH); }
uint32_t scan_tiles_x(uint32_t w) { return (w + kTW - 1) / kTW; }

void scan_encode_batch(const BatchScanFrame* frames, uint32_t n_frames, uint32_t n_tiles, int r1, int r2,
                       uint32_t ctas, cudaStream_t s) {
    if (n_tiles == 0) return;
    Probe p("scan_encode_batch", s);
    if (r1 == 5 && r2 == 2) launch_scan_batch<5, 2>(frames, n_frames, n_tiles, ctas, scan_smem_bytes(5, 2), s);
    else launch_scan_batch<-1, -1>(frames, n_frames, n_tiles, ctas, scan_smem_bytes(SPKB_FIR_MAX_R, SPKB_FIR_MAX_R), s);
}

namespace {
template <int R>
void launch_fir_tile(const float* in, float* out, uint32_t w, uint32_t h, const ScanArgs& a, cudaStream_t s) {
    const size_t smem = size_t(2 * kTH + 2 * a.r1) * size_t(3 * (kTW + 2 * a.r1)) * sizeof(float);
    ensure_smem(reinterpret_cast<const void*>(k_fir_tile<R>), int(smem));
    const dim3 g((w + kTW - 1) / kTW, (h + kTH - 1) / kTH);
    k_fir_tile<R><<<g, kThreads, smem, s>>>(in, out, int(w), int(h), a);
}
}  // namespace

bool fir_tile_fits(uint32_t w, uint32_t h, int r) { return scan_encode_fits(w, h, r, 0); }

void fir_tile(const float* in, float* out, uint32_t w, uint32_t h, int r, const float* taps, cudaStream_t s) {
    if (uint64_t(w) * h == 0) return;
    ScanArgs a{};
    a.r1 = r;
    for (int k = 0; k <= 2 * r; ++k) a.t1[k] = taps[k];
    Probe p("fir_tile", s);
    if (r == 2) launch_fir_tile<2>(in, out, w, h, a, s);
    else if (r == 5) launch_fir_tile<5>(in, out, w, h, a, s);
    else launch_fir_tile<-1>(in, out, w, h, a, s);
}

}  // namespace spkb::dev
