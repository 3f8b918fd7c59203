// The tier downscale and the decode + geometry stage: binary64 set-up on the host, the passes on the
// device (csrc/cuda/prepare.cu).
#include "tiers.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../cuda/launch.hpp"
#include "resources.hpp"
#include "setup.hpp"
#include "status.hpp"

namespace spkb {

Size2 downscale_size(uint32_t w, uint32_t h, uint32_t long_edge) {
    const uint32_t m = std::max(w, h);
    if (long_edge == 0 || m <= long_edge) return {w, h};
    const double s = double(long_edge) / double(m);
    const double fw = std::floor(double(w) * s), fh = std::floor(double(h) * s);
    return {std::max<uint32_t>(1, uint32_t(fw)), std::max<uint32_t>(1, uint32_t(fh))};
}

std::vector<float> tier_axis_taps(uint32_t n, uint32_t m) {
    const double sigma = std::max(0.0, (double(n) / double(m) - 1.0) / 2.0);
    const std::vector<double> w = gaussian_kernel(sigma, 4.0);
    std::vector<float> f(w.size());
    for (size_t i = 0; i < w.size(); ++i) f[i] = f32(w[i]);
    return f;
}

// The source coordinate (o + 1/2) n / m - 1/2 is num / den with num = (2 o + 1) n - m and den = 2 m,
// mirrored at both ends into [0, n - 1] (reference src/session/tiers.cpp:66-97).
TierAxisSamples tier_axis_samples(uint32_t n, uint32_t m) {
    TierAxisSamples s;
    s.idx.resize(size_t(2) * m);
    s.t.resize(m);
    const int64_t N = n, M = m, den = 2 * M;
    for (int64_t o = 0; o < M; ++o) {
        int64_t num = (2 * o + 1) * N - M;
        if (num > den * (N - 1)) num = 2 * den * (N - 1) - num;
        if (num < 0) num = -num;
        const int64_t i0 = std::min<int64_t>(num / den, N - 1);
        const int64_t i1 = std::min<int64_t>(i0 + 1, N - 1);
        s.idx[size_t(2 * o)] = uint32_t(i0);
        s.idx[size_t(2 * o + 1)] = uint32_t(i1);
        s.t[size_t(o)] = float(num - i0 * den) / float(den);
    }
    return s;
}

Plane downscale(Pool& pool, cudaStream_t s, const Plane& src, uint32_t long_edge) {
    const Size2 o = downscale_size(src.w, src.h, long_edge);
    if (o.w == src.w && o.h == src.h) return src;
    const std::vector<float> ty = tier_axis_taps(src.h, o.h), tx = tier_axis_taps(src.w, o.w);
    const TierAxisSamples sx = tier_axis_samples(src.w, o.w), sy = tier_axis_samples(src.h, o.h);
    // one upload of every table: taps y | taps x | xi | xt | yi | yt (4-byte words)
    std::vector<uint32_t> words;
    auto put = [&](const void* p, size_t n) {
        const size_t at = words.size();
        words.resize(at + n);
        std::memcpy(words.data() + at, p, n * 4);
        return at;
    };
    const size_t oty = put(ty.data(), ty.size()), otx = put(tx.data(), tx.size());
    const size_t oxi = put(sx.idx.data(), sx.idx.size()), oxt = put(sx.t.data(), sx.t.size());
    const size_t oyi = put(sy.idx.data(), sy.idx.size()), oyt = put(sy.t.data(), sy.t.size());
    DevBuffer tab = pool.acquire(words.size() * 4);
    cuda_check(cudaMemcpyAsync(tab.ptr(), words.data(), words.size() * 4, cudaMemcpyHostToDevice, s), "tier tables");
    const uint32_t* base = tab.as<uint32_t>();

    Plane v = src;
    Plane vb;
    if (ty.size() > 1) {
        vb = make_plane(pool, src.w, src.h);
        TierBlurArgs a{reinterpret_cast<const float*>(base + oty), src.w, src.h, int32_t(ty.size() / 2)};
        dev::tier_blur_v(src.data(), vb.data(), a, s);
        v = vb;
    }
    Plane out;
    out.w = o.w;
    out.h = o.h;
    out.buf = pool.persistent(size_t(o.w) * o.h * 3 * sizeof(float));
    TierResampleArgs r{};
    r.taps_x = reinterpret_cast<const float*>(base + otx);
    r.xi = base + oxi;
    r.xt = reinterpret_cast<const float*>(base + oxt);
    r.yi = base + oyi;
    r.yt = reinterpret_cast<const float*>(base + oyt);
    r.in_w = src.w;
    r.in_h = src.h;
    r.out_w = o.w;
    r.out_h = o.h;
    r.rx = int32_t(tx.size() / 2);
    dev::tier_resample(v.data(), out.data(), r, s);
    cuda_check(cudaStreamSynchronize(s), "tier downscale");  // the host tables go out of scope
    return out;
}

bool geometry_identity(const ParamSet& p) {
    return p.f(P::geometry_crop_x) == 0.0 && p.f(P::geometry_crop_y) == 0.0 && p.f(P::geometry_crop_w) == 1.0 &&
           p.f(P::geometry_crop_h) == 1.0 && p.f(P::geometry_rotation_deg) == 0.0 &&
           ((p.i(P::geometry_quarter_turns) % 4) + 4) % 4 == 0 && !p.b(P::geometry_flip_h) && !p.b(P::geometry_flip_v);
}

namespace {

struct GeometryScalars {
    uint32_t q = 0;
    bool fh = false, fv = false;
    double sx = 0, sy = 0, hx = 0, hy = 0, ca = 1, sa = 0, ow = 0, oh = 0, cx = 0, cy = 0;
};

// The binary64 constants of the geometry (reference src/film/geometry.cpp:45-82); the output size is
// the rounded crop, its sides exchanged by an odd quarter turn.
GeometryScalars geometry_scalars(const ParamSet& p, uint32_t SW, uint32_t SH, uint32_t& dst_w, uint32_t& dst_h) {
    GeometryScalars g;
    const double cx = p.f(P::geometry_crop_x), cy = p.f(P::geometry_crop_y);
    const double cw = p.f(P::geometry_crop_w), ch = p.f(P::geometry_crop_h);
    g.q = uint32_t(((p.i(P::geometry_quarter_turns) % 4) + 4) % 4);
    g.fh = p.b(P::geometry_flip_h);
    g.fv = p.b(P::geometry_flip_v);
    const double CW = std::max(1.0, std::round(cw * double(SW)));
    const double CH = std::max(1.0, std::round(ch * double(SH)));
    const bool odd = (g.q & 1u) != 0;
    g.ow = odd ? CH : CW;
    g.oh = odd ? CW : CH;
    dst_w = uint32_t(g.ow);
    dst_h = uint32_t(g.oh);
    g.sx = cw * double(SW) / CW;
    g.sy = ch * double(SH) / CH;
    g.hx = cw * double(SW) / 2.0;
    g.hy = ch * double(SH) / 2.0;
    g.cx = (cx + cw / 2.0) * double(SW) - 0.5;
    g.cy = (cy + ch / 2.0) * double(SH) - 0.5;
    const double theta = p.f(P::geometry_rotation_deg) * 3.14159265358979323846 / 180.0;
    g.ca = std::cos(theta);
    g.sa = std::sin(theta);
    return g;
}

}  // namespace

Size2 prepared_size(const ParamSet& p, uint32_t w, uint32_t h) {
    if (geometry_identity(p)) return {w, h};
    Size2 o;
    geometry_scalars(p, w, h, o.w, o.h);
    return o;
}

Plane prepare_source(Pool& pool, cudaStream_t s, const Plane& src, const ParamSet& p, bool decode, uint32_t cctf_mode) {
    const bool geometry = !geometry_identity(p);
    if (!decode && !geometry) return src;
    PrepareArgs a{};
    a.decode = decode ? 1 : 0;
    a.mode = cctf_mode;
    a.bt709_bp = f32(1.099 * std::pow(0.018, 0.45) - 0.099);
    a.bt709_exp = f32(1.0 / 0.45);
    a.geometry = geometry ? 1 : 0;
    a.src_w = src.w;
    a.src_h = src.h;
    a.dst_w = src.w;
    a.dst_h = src.h;
    if (geometry) {
        const GeometryScalars k = geometry_scalars(p, src.w, src.h, a.dst_w, a.dst_h);
        a.quarter = k.q;
        a.flip_h = k.fh ? 1u : 0u;
        a.flip_v = k.fv ? 1u : 0u;
        a.sx = k.sx;
        a.sy = k.sy;
        a.hx = k.hx;
        a.hy = k.hy;
        a.ca = k.ca;
        a.sa = k.sa;
        a.ow = k.ow;
        a.oh = k.oh;
        a.cx = k.cx;
        a.cy = k.cy;
    }
    Plane out = make_plane(pool, a.dst_w, a.dst_h);
    dev::prepare(src.data(), out.data(), a, s);
    return out;
}

}  // namespace spkb
