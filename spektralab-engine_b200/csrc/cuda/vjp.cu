// The adjoint of the render path's per-pixel stages and of the FIR passes (declarations in vjp.hpp).
//
// Every per-pixel stage is re-evaluated on dual numbers with one tangent per input channel (and, for the
// print stage, per print-side parameter); its formulas and bracketing are those of the forward kernels
// (kernels.cu, print.cu) and of the reference (kernels/film.metal, fx_grain.metal, print.metal), with the
// accurate binary32 library functions throughout. The vector-Jacobian product is then the upstream
// gradient contracted with the tangents.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "dual.cuh"
#include "launch.hpp"
#include "lookup.cuh"
#include "vjp.hpp"

namespace spkb::dev {

namespace {

constexpr float kTinyV = 1e-10f;

// ---- expose (reference kernels/film.metal:50-99, :189-227) ------------------------------------------

template <int N>
__device__ __forceinline__ Dual<N> mitchell_d(const Dual<N>& u) {
    const Dual<N> a = dfabs(u);
    if (a.v < 1.0f) return (1.0f / 6.0f) * (((7.0f * a) * a) * a - (12.0f * a) * a + 16.0f / 3.0f);
    if (a.v < 2.0f)
        return (1.0f / 6.0f) * ((((-7.0f / 3.0f) * a) * a) * a + (12.0f * a) * a - 20.0f * a + 32.0f / 3.0f);
    return dconst<N>(0.0f);
}

template <int N>
__device__ __forceinline__ void mitchell_axis_d(const Dual<N>& t, uint32_t L, int* idx, Dual<N>* w) {
    const float last = float(L - 1);
    Dual<N> u = t * last;
    int base;
    Dual<N> frac;
    if (u.v <= 0.0f) u = dconst<N>(0.0f);
    if (u.v >= last) {
        base = int(L) - 2;
        frac = dconst<N>(1.0f);
    } else {
        base = int(floorf(u.v));
        frac = u - float(base);
    }
    const int n = int(L);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int i = base - 1 + k;
        if (i < 0) i = -i;
        if (i >= n) i = 2 * (n - 1) - i;
        idx[k] = i;
    }
    w[0] = mitchell_d(frac + 1.0f);
    w[1] = mitchell_d(frac);
    w[2] = mitchell_d(frac - 1.0f);
    w[3] = mitchell_d(frac - 2.0f);
}

__global__ void k_vjp_expose(const float* __restrict__ rgb, const float* __restrict__ g_h, float* __restrict__ g_rgb,
                             const float4* __restrict__ table, const __grid_constant__ ExposeArgs q) {
    using D3 = Dual<3>;
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= q.n) return;
    const size_t o3 = 3 * size_t(gid);
    const D3 r = dvar<3>(rgb[o3], 0), g = dvar<3>(rgb[o3 + 1], 1), b = dvar<3>(rgb[o3 + 2], 2);
    const D3 X = (q.a[0] * r + q.a[1] * g) + q.a[2] * b;
    const D3 Y = (q.a[3] * r + q.a[4] * g) + q.a[5] * b;
    const D3 Z = (q.a[6] * r + q.a[7] * g) + q.a[8] * b;
    const D3 bs = (X + Y) + Z;
    const D3 d = bs.v > 1e-10f ? bs : dconst<3>(1e-10f);
    const D3 x = X / d, y = Y / d, o = 1.0f - x;
    const D3 t0 = dclamp(o * o, 0.0f, 1.0f);
    const D3 t1 = dclamp(y / (o.v > 1e-10f ? o : dconst<3>(1e-10f)), 0.0f, 1.0f);
    const D3 bp = isnan(bs.v) ? dconst<3>(0.0f) : bs;
    int ia[4], ib[4];
    D3 wa[4], wb[4];
    mitchell_axis_d(t0, q.L, ia, wa);
    mitchell_axis_d(t1, q.L, ib, wb);
    D3 s = dconst<3>(0.0f), a0 = s, a1 = s, a2 = s;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            const D3 wgt = wa[i] * wb[j];
            const float4 t = __ldg(table + (size_t(ia[i]) * q.L + size_t(ib[j])));
            s = s + wgt;
            a0 = a0 + wgt * t.x;
            a1 = a1 + wgt * t.y;
            a2 = a2 + wgt * t.z;
        }
    if (s.v != 0.0f) {
        a0 = a0 / s;
        a1 = a1 / s;
        a2 = a2 / s;
    }
    D3 h[3] = {bp * a0, bp * a1, bp * a2};
    if (q.apply_gain)
        for (int c = 0; c < 3; ++c) h[c] = h[c] * q.gain;
    const float gh[3] = {g_h[o3], g_h[o3 + 1], g_h[o3 + 2]};
#pragma unroll
    for (int i = 0; i < 3; ++i) g_rgb[o3 + i] = (gh[0] * h[0].d[i] + gh[1] * h[1].d[i]) + gh[2] * h[2].d[i];
}

// ---- develop, grain as fixed noise (reference kernels/film.metal:242-261, fx_grain.metal:39-97) ------

// the hat functions of the density-curve parameters at table entry k: phi_j(k) (1 - f) and phi_{j+1}(k) f
__device__ __forceinline__ void curve_basis(uint32_t k, uint32_t K, uint32_t& j, float& f) {
    const float u = float(k) * (float(kVjpCurveNodes - 1) / float(K - 1));
    j = min(uint32_t(u), uint32_t(kVjpCurveNodes - 2));
    f = u - float(j);
}

__global__ void k_vjp_develop(const float* __restrict__ exposure, const float* __restrict__ counts,
                              const float* __restrict__ g_neg, float* __restrict__ g_exp, double* __restrict__ g_nodes,
                              uint32_t w, uint32_t h, const __grid_constant__ DevelopArgs q) {
    using D2 = Dual<2>;  // tangents: the exposure, and the density the curve returns
    __shared__ float acc[3 * kVjpCurveNodes];
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    if (g_nodes) {
        for (uint32_t i = tid; i < 3u * kVjpCurveNodes; i += nt) acc[i] = 0.0f;
        __syncthreads();
    }
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < w && y < h) {
        const uint32_t pixel = y * q.width + x;
        const size_t o = 3 * (size_t(y) * w + x);
        for (uint32_t c = 0; c < 3; ++c) {
            const D2 H = dvar<2>(exposure[o + c], 0);
            const D2 L = dlog10(dfmax(H, 0.0f) + 1e-10f);
            // the curve lookup (reference kernels/film.metal:84-101), keeping its interval l and fraction t
            const float* cy = q.cy + size_t(c) * q.K;
            D2 D;
            uint32_t l = 0;
            float t = 0.0f;
            if (L.v <= __ldg(q.cx)) {
                D = dconst<2>(__ldg(cy));
            } else if (L.v >= __ldg(q.cx + q.K - 1)) {
                D = dconst<2>(__ldg(cy + q.K - 1));
                l = q.K - 2;
                t = 1.0f;
            } else {
                l = axis_index(q.cx, 1, q.K, q.cgrid, L.v);
                const D2 td = (L - __ldg(q.cx + l)) * __ldg(q.cinv + l);
                const float y0 = __ldg(cy + l);
                D = y0 + td * (__ldg(cy + l + 1) - y0);
                t = td.v;
            }
            D.d[1] = 1.0f;
            D2 out = D;
            if (q.grain) {
                const D2 v = q.positive ? -D : D;
                const uint32_t K = q.gK;
                D2 dl[3];
                if (v.v <= __ldg(q.axis + c)) {
                    for (uint32_t k = 0; k < 3u; ++k) dl[k] = dconst<2>(__ldg(q.layers + k * 3u + c));
                } else if (v.v >= __ldg(q.axis + 3u * (K - 1u) + c)) {
                    for (uint32_t k = 0; k < 3u; ++k) dl[k] = dconst<2>(__ldg(q.layers + ((K - 1u) * 3u + k) * 3u + c));
                } else {
                    const uint32_t j = axis_index(q.axis + c, 3u, K, q.ggrid[c], v.v);
                    const D2 tg = (v - __ldg(q.axis + 3u * j + c)) * __ldg(q.ginv + 3u * j + c);
                    for (uint32_t k = 0; k < 3u; ++k) {
                        const float y0 = __ldg(q.layers + (j * 3u + k) * 3u + c);
                        const float y1 = __ldg(q.layers + ((j + 1u) * 3u + k) * 3u + c);
                        dl[k] = y0 + tg * (y1 - y0);
                    }
                }
                D2 G = dconst<2>(0.0f);
                for (uint32_t k = 0; k < 3u; ++k) {
                    const uint32_t lc = k * 3u + c;
                    const D2 qd = dclamp((dl[k] + q.dmin_l[lc]) / q.sat_d[lc], 1e-6f, 0.999999f);
                    const D2 sat = 1.0f - (qd * q.uniformity[c]) * 0.999999f;
                    const float cnt = counts[size_t(pixel) * 9 + c * 3 + k];
                    G = G + cnt * ((q.sat_d[lc] / q.count[lc]) * sat);
                }
                if (q.shift) G = G + (-q.dmin_c[c]);
                out = G;
            }
            const float gn = g_neg[o + c];
            g_exp[o + c] = gn * out.d[0];
            if (g_nodes) {
                const float gd = gn * out.d[1];
                if (gd != 0.0f) {
                    uint32_t j;
                    float f;
                    curve_basis(l, q.K, j, f);
                    atomicAdd(&acc[c * kVjpCurveNodes + j], gd * (1.0f - t) * (1.0f - f));
                    atomicAdd(&acc[c * kVjpCurveNodes + j + 1], gd * (1.0f - t) * f);
                    if (t != 0.0f) {
                        curve_basis(l + 1, q.K, j, f);
                        atomicAdd(&acc[c * kVjpCurveNodes + j], gd * t * (1.0f - f));
                        atomicAdd(&acc[c * kVjpCurveNodes + j + 1], gd * t * f);
                    }
                }
            }
        }
    }
    if (g_nodes) {
        __syncthreads();
        for (uint32_t i = tid; i < 3u * kVjpCurveNodes; i += nt)
            if (acc[i] != 0.0f) atomicAdd(g_nodes + i, double(acc[i]));
    }
}

// ---- print (reference kernels/print.metal:29-127, :165-317) ------------------------------------------

constexpr int NP = 3 + kVjpPrintParams;  // tangents: the three negative densities, then the parameters
using DP = Dual<NP>;


// R_k = sum_l 10^-(d . eps(l) + beta(l)) wt_k(l), ascending l, with its tangents written out rather than
// carried through dual products (most of a dual product's terms are zero here): per wavelength
//   x = d . eps + beta,  x' = d' . eps + d . eps' + beta',  T = 10^-x,  T' = -ln(10) T x',
//   R_k += T wt_k,  R_k' += T' wt_k + T wt_k'
// with eps', beta', wt' the print parameters' tangents (components 3..; none where t_* is null), each
// stored [parameter][index] with the strides of the tables.
__device__ void spectral_d(const float* eps, const float* beta, const float* wt, const float* t_eps,
                           const float* t_beta, const float* t_wt, const DP* d, DP* R) {
    float r[3] = {0.0f, 0.0f, 0.0f};
    float rd[3][NP];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < NP; ++i) rd[k][i] = 0.0f;
#pragma unroll 3
    for (int l = 0; l < SPKB_NL; ++l) {
        const float e0 = eps[3 * l], e1 = eps[3 * l + 1], e2 = eps[3 * l + 2];
        const float x = ((d[0].v * e0 + d[1].v * e1) + d[2].v * e2) + beta[l];
        float xd[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) xd[i] = (d[0].d[i] * e0 + d[1].d[i] * e1) + d[2].d[i] * e2;
        if (t_eps) {
#pragma unroll
            for (int j = 0; j < kVjpPrintParams; ++j) {
                const float* te = t_eps + j * 3 * SPKB_NL + 3 * l;
                xd[3 + j] += ((d[0].v * te[0] + d[1].v * te[1]) + d[2].v * te[2]) + t_beta[j * SPKB_NL + l];
            }
        }
        const float T = exp10f(-x);
        const float cT = -2.30258509299404568f * T;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float wk = wt[3 * l + k];
            r[k] += T * wk;
            const float cw = cT * wk;
#pragma unroll
            for (int i = 0; i < NP; ++i) rd[k][i] += cw * xd[i];
            if (t_wt) {
#pragma unroll
                for (int j = 0; j < kVjpPrintParams; ++j) rd[k][3 + j] += T * t_wt[j * 3 * SPKB_NL + 3 * l + k];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R[k].v = r[k];
#pragma unroll
        for (int i = 0; i < NP; ++i) R[k].d[i] = rd[k][i];
    }
}

__device__ __forceinline__ DP paper_d(const VjpPrintArgs& a, uint32_t c, const DP& v) {
    if (isnan(v.v)) return v;
    const uint32_t K = a.paper_K;
    const float* x = a.paper;
    const float* r = a.paper + K;
    const float* y = a.paper + 2 * K;
    if (v.v <= __ldg(x)) return dconst<NP>(__ldg(y + c));
    if (v.v >= __ldg(x + K - 1)) return dconst<NP>(__ldg(y + 3 * (K - 1) + c));
    const uint32_t j = axis_index(x, 1, K, a.paper_grid, v.v);
    const float y0 = __ldg(y + 3 * j + c);
    return y0 + ((v - __ldg(x + j)) * __ldg(r + j)) * (__ldg(y + 3 * (j + 1) + c) - y0);
}

__device__ __forceinline__ DP knee_d(const DP& d, float tau, float lim, float p) {
    if (d.v <= tau) return d;
    const DP x = (d - tau) / (lim - tau);
    return tau + (lim - tau) * (x / dpow(1.0f + dpow(x, p), 1.0f / p));
}

__device__ __forceinline__ DP post_adapt_d(const DP& v, float f_l) {
    const DP f = dpow((f_l * dfabs(v)) / 100.0f, 0.42f);
    return ((400.0f * dsgn(v)) * f) / (27.13f + f) + 0.1f;
}

// CAM16-UCS gamut compression, the forward kernel's formulas on duals
__device__ void gamut_d(const VjpPrintArgs& pa, DP& r, DP& g, DP& b) {
    const Cam16Args& q = pa.cam;
    const float cz = q.cz, inv_cz = q.inv_cz, f_l_qrt = q.f_l_qrt, chroma_k = q.chroma_k;
    DP X, Y, Z;
    dmat(q.m_to_xyz, r, g, b, X, Y, Z);
    DP R16, G16, B16;
    dmat(q.m16, 100.0f * X, 100.0f * Y, 100.0f * Z, R16, G16, B16);
    const DP ra = post_adapt_d(q.d_rgb[0] * R16, q.f_l);
    const DP ga = post_adapt_d(q.d_rgb[1] * G16, q.f_l);
    const DP ba = post_adapt_d(q.d_rgb[2] * B16, q.f_l);
    const DP a = (ra - (12.0f * ga) / 11.0f) + ba / 11.0f;
    const DP bb = ((ra + ga) - 2.0f * ba) / 9.0f;
    const DP h = datan2(bb, a);
    const DP et = 0.25f * (dcos(h + 2.0f) + 3.8f);
    const DP A = (((2.0f * ra + ga) + ba / 20.0f) - 0.305f) * q.n_bb;
    const DP ratio = A / q.a_w;
    const DP J = (100.0f * dsgn(ratio)) * dpow(dfabs(ratio), cz);
    const DP den = (ra + ga) + (21.0f * ba) / 20.0f;
    const DP t = den.v != 0.0f
                     ? (((((50000.0f / 13.0f) * q.n_c) * q.n_cb) * et) * dsqrt(a * a + bb * bb)) / den
                     : dconst<NP>(0.0f);
    const DP C = t.v > 0.0f ? (dpow(t, 0.9f) * dsqrt(dfabs(J) / 100.0f)) * chroma_k : dconst<NP>(0.0f);
    const DP M = C * f_l_qrt;
    const DP Mp = dlog(1.0f + 0.0228f * M) / 0.0228f;
    DP Jp = (1.7f * J) / (1.0f + 0.007f * J);
    if (q.lc_active != 0u) {
        DP Ln = Jp / q.j_white;
        if (Ln.v > q.lc[0]) {
            Ln = knee_d(Ln, q.lc[0], q.lc[1], q.lc[2]);
            Jp = Ln * q.j_white;
        }
    }
    const DP Jc = dclamp(Jp, q.j_first, q.j_last);
    const DP u = ((Jc - q.j_first) / (q.j_last - q.j_first)) * float(q.rows - 1);
    int l0 = int(floorf(u.v));
    l0 = l0 < 0 ? 0 : (l0 > int(q.rows) - 2 ? int(q.rows) - 2 : l0);
    const DP fl = u - float(l0);
    const DP v = (h - q.h_first) / q.h_step;
    const float vf = floorf(v.v);
    const int cols = int(q.cols);
    int h0 = int(vf) % cols;
    if (h0 < 0) h0 += cols;
    const int h1 = h0 == cols - 1 ? 0 : h0 + 1;
    const DP fh = v - vf;
    const float t00 = __ldg(pa.cmax + l0 * cols + h0), t01 = __ldg(pa.cmax + l0 * cols + h1);
    const float t10 = __ldg(pa.cmax + (l0 + 1) * cols + h0), t11 = __ldg(pa.cmax + (l0 + 1) * cols + h1);
    const DP cm = (1.0f - fl) * ((1.0f - fh) * t00 + fh * t01) + fl * ((1.0f - fh) * t10 + fh * t11);
    const DP cs = dfmax(cm, 1e-9f);
    DP dch = Mp / cs;
    if (dch.v > 0.0f) dch = knee_d(dch, q.knee[0], q.knee[1], q.knee[2]);
    const DP Mn = dch * cs;
    const DP Mi = (dexp(0.0228f * Mn) - 1.0f) / 0.0228f;
    const DP Ji = Jp / (1.7f - 0.007f * Jp);
    const DP Ci = Mi / f_l_qrt;
    const DP Ai = (q.a_w * dsgn(Ji)) * dpow(dfabs(Ji / 100.0f), inv_cz);
    const DP sq = dsqrt(dfabs(Ji) / 100.0f);
    const DP ti = (sq.v > 0.0f && Ci.v > 0.0f) ? dpow(Ci / (sq * chroma_k), 1.0f / 0.9f) : dconst<NP>(0.0f);
    const DP p2 = Ai / q.n_bb + 0.305f;
    const float p3 = 21.0f / 20.0f;
    DP ai = dconst<NP>(0.0f), bi = dconst<NP>(0.0f);
    if (ti.v != 0.0f) {
        const DP p1 = ((((50000.0f / 13.0f) * q.n_c) * q.n_cb) * et) / ti;
        const DP sh = dsin(h), ch = dcos(h);
        if (fabsf(sh.v) >= fabsf(ch.v)) {
            const DP p4 = p1 / sh;
            bi = ((p2 * (2.0f + p3)) * (460.0f / 1403.0f)) /
                 (((p4 + ((2.0f + p3) * (220.0f / 1403.0f)) * (ch / sh)) - 27.0f / 1403.0f) + p3 * (6300.0f / 1403.0f));
            ai = (bi * ch) / sh;
        } else {
            const DP p5 = p1 / ch;
            ai = ((p2 * (2.0f + p3)) * (460.0f / 1403.0f)) /
                 ((p5 + (2.0f + p3) * (220.0f / 1403.0f)) - (27.0f / 1403.0f - p3 * (6300.0f / 1403.0f)) * (sh / ch));
            bi = (ai * sh) / ch;
        }
    }
    const DP xa[3] = {((460.0f * p2 + 451.0f * ai) + 288.0f * bi) / 1403.0f,
                      ((460.0f * p2 - 891.0f * ai) - 261.0f * bi) / 1403.0f,
                      ((460.0f * p2 - 220.0f * ai) - 6300.0f * bi) / 1403.0f};
    DP rc[3];
    for (int i = 0; i < 3; ++i) {
        const DP vv = xa[i] - 0.1f;
        const DP av = dfabs(vv);
        const DP beta = av.v >= 400.0f ? dconst<NP>(0.0f) : (27.13f * av) / (400.0f - av);
        rc[i] = ((q.hundred_over_f_l * dsgn(vv)) * dpow(beta, 1.0f / 0.42f)) / q.d_rgb[i];
    }
    DP x100, y100, z100;
    dmat(q.m16_inv, rc[0], rc[1], rc[2], x100, y100, z100);
    dmat(q.m_to_rgb, x100 / 100.0f, y100 / 100.0f, z100 / 100.0f, r, g, b);
}

// threads per CTA of the print's adjoint (VJP at 1024x1024: 5.02 ms at 128, 4.64 at 256, 5.91 at 512)
#ifndef SPKB_VJP_PRINT_THREADS
#define SPKB_VJP_PRINT_THREADS 256
#endif
constexpr uint32_t kVjpPrintThreads = SPKB_VJP_PRINT_THREADS;

__global__ void __launch_bounds__(kVjpPrintThreads) k_vjp_print(const float* __restrict__ neg, const float* __restrict__ g_p,
                                                   float* __restrict__ g_neg, double* __restrict__ grad_params,
                                                   const __grid_constant__ VjpPrintArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double part[kVjpPrintParams] = {0.0, 0.0, 0.0};
    if (i < a.n) {
        const size_t o = 3 * size_t(i);
        DP d[3] = {dvar<NP>(neg[o], 0), dvar<NP>(neg[o + 1], 1), dvar<NP>(neg[o + 2], 2)};
        if (a.printed) {
            DP R[3];
            spectral_d(a.enl_eps, a.enl_beta, a.enl_wt, &a.t_eps[0][0], &a.t_beta[0][0], &a.t_wt[0][0], d, R);
            for (uint32_t c = 0; c < 3; ++c) {
                DP gc = dconst<NP>(a.g[c]), oc = dconst<NP>(a.o[c]), kg = dconst<NP>(a.k_gain);
                for (int j = 0; j < kVjpPrintParams; ++j) {
                    gc.d[3 + j] = a.t_g[j][c];
                    oc.d[3 + j] = a.t_o[j][c];
                    kg.d[3 + j] = a.t_k[j];
                }
                DP l = dlog10(dfmax(R[c] * gc + oc, 0.0f) + kTinyV);
                l = dlog10(dfmax(dexp10(l) * kg, 0.0f) + kTinyV);
                d[c] = paper_d(a, c, l);
            }
        }
        DP S[3];
        spectral_d(a.scan_eps, a.scan_beta, a.scan_wt, nullptr, nullptr, nullptr, d, S);
        for (int c = 0; c < 3; ++c) S[c] = dfmax(S[c], 0.0f) + kTinyV;
        DP r, g, b;
        dmat(a.to_rgb, S[0], S[1], S[2], r, g, b);
        gamut_d(a, r, g, b);
        const float gp[3] = {g_p[o], g_p[o + 1], g_p[o + 2]};
#pragma unroll
        for (int k = 0; k < 3; ++k) g_neg[o + k] = (gp[0] * r.d[k] + gp[1] * g.d[k]) + gp[2] * b.d[k];
#pragma unroll
        for (int j = 0; j < kVjpPrintParams; ++j)
            part[j] = (double(gp[0]) * r.d[3 + j] + double(gp[1]) * g.d[3 + j]) + double(gp[2]) * b.d[3 + j];
    }
    // one binary64 atomic per warp and parameter
#pragma unroll
    for (int j = 0; j < kVjpPrintParams; ++j) {
        double v = part[j];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
        if ((threadIdx.x & 31u) == 0u) atomicAdd(grad_params + j, v);
    }
}

// ---- FIR pass transpose (reference kernels/fx_blur.metal:20-78) --------------------------------------
//
// A pass out[i] = sum_k t[k] in[refl(i + k - r)] along a line of n samples (refl: half-sample symmetric,
// exact for the offsets here since n > r). Its transpose gathers, for sample j, every (i, k) whose tap
// lands on j: i + k - r is one of j, -1 - j (reflected off the start) and 2n - 1 - j (off the end).
__global__ void k_fir_pass_adj(const float* __restrict__ g_out, float* __restrict__ g_in, int w, int h, int r,
                               const __grid_constant__ FirTaps t, int vertical) {
    const int x = int(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = int(blockIdx.y * blockDim.y + threadIdx.y);
    if (x >= w || y >= h) return;
    const int n = vertical ? h : w, j = vertical ? y : x;
    const size_t step = vertical ? size_t(w) * 3 : 3;
    const float* line = g_out + (vertical ? size_t(x) * 3 : size_t(y) * w * 3);
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    const int pre[3] = {j, -1 - j, 2 * n - 1 - j};
    for (int m = 0; m < 3; ++m) {
        for (int k = 0; k <= 2 * r; ++k) {
            const int i = pre[m] - k + r;
            if (i < 0 || i >= n) continue;
            const float* p = line + size_t(i) * step;
            a0 += t.taps[0][k] * p[0];
            a1 += t.taps[1][k] * p[1];
            a2 += t.taps[2][k] * p[2];
        }
    }
    float* o = g_in + 3 * (size_t(y) * w + x);
    o[0] = a0;
    o[1] = a1;
    o[2] = a2;
}

__global__ void k_dot3(const float* __restrict__ x, const float* __restrict__ y, size_t pixels, double* acc) {
    double s[3] = {0.0, 0.0, 0.0};
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < pixels; p += size_t(gridDim.x) * blockDim.x)
        for (int c = 0; c < 3; ++c) s[c] += double(x[3 * p + c]) * double(y[3 * p + c]);
    for (int c = 0; c < 3; ++c) {
        double v = s[c];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
        if ((threadIdx.x & 31u) == 0u) atomicAdd(acc + c, v);
    }
}

}  // namespace

void vjp_print(const float* neg, const float* g_print, float* g_neg, double* grad_params, const VjpPrintArgs& a,
               cudaStream_t s) {
    if (a.n == 0) return;
    Probe p("vjp_print", s);
    k_vjp_print<<<(a.n + kVjpPrintThreads - 1) / kVjpPrintThreads, kVjpPrintThreads, 0, s>>>(neg, g_print, g_neg,
                                                                                             grad_params, a);
}

void vjp_develop(const float* exposure, const float* counts, const float* g_neg, float* g_exposure,
                 double* g_nodes, const DevelopArgs& a, uint32_t w, uint32_t h, cudaStream_t s) {
    if (uint64_t(w) * h == 0) return;
    const dim3 b(32, 4), g((w + 31) / 32, (h + 3) / 4);
    Probe p("vjp_develop", s);
    k_vjp_develop<<<g, b, 0, s>>>(exposure, counts, g_neg, g_exposure, g_nodes, w, h, a);
}

void vjp_expose(const float* rgb, const float* g_h, float* g_rgb, const float* table4, const ExposeArgs& a,
                cudaStream_t s) {
    if (a.n == 0) return;
    Probe p("vjp_expose", s);
    k_vjp_expose<<<(a.n + 127) / 128, 128, 0, s>>>(rgb, g_h, g_rgb, reinterpret_cast<const float4*>(table4), a);
}

void fir_pass_adjoint(const float* g_out, float* g_in, uint32_t w, uint32_t h, int r, const float* taps,
                      int vertical, cudaStream_t s) {
    if (uint64_t(w) * h == 0) return;
    FirTaps t{};
    t.r = r;
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k <= 2 * r; ++k) t.taps[c][k] = taps[k];
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    Probe p("fir_pass_adjoint", s);
    k_fir_pass_adj<<<g, b, 0, s>>>(g_out, g_in, int(w), int(h), r, t, vertical);
}

void dot3(const float* x, const float* y, size_t pixels, double* acc, cudaStream_t s) {
    if (pixels == 0) return;
    Probe p("dot3", s);
    k_dot3<<<148 * 4, 256, 0, s>>>(x, y, pixels, acc);
}

}  // namespace spkb::dev
