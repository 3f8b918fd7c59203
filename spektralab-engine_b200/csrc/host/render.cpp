#include "render.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "../cuda/iir.hpp"
#include "../cuda/launch.hpp"
#include "../cuda/vjp.hpp"
#include "blur_plan.h"
#include "status.hpp"
#include "tiers.hpp"

namespace spkb {

namespace {

void upload(Pool& pool, cudaStream_t s, DevBuffer& dst, const void* src, size_t bytes) {
    dst = pool.persistent(bytes);
    cuda_check(cudaMemcpyAsync(dst.ptr(), src, bytes, cudaMemcpyHostToDevice, s), "table upload");
}

}  // namespace

void upload_tables(Pool& pool, cudaStream_t s, Pipeline& p) {
    const FilmSetup& f = *p.film;
    {
        // the spectral table as 16-byte texels (R, G, B, 0): one vector load per bicubic tap
        const size_t texels = f.table32.size() / 3;
        std::vector<float> t4(4 * texels, 0.0f);
        for (size_t i = 0; i < texels; ++i)
            for (size_t c = 0; c < 3; ++c) t4[4 * i + c] = f.table32[3 * i + c];
        upload(pool, s, p.dev.table, t4.data(), t4.size() * sizeof(float));
        // the 4 x 4 patch of every base pair (ba, bb): rows and columns base - 1 .. base + 2, reflected at
        // the table's edges as the bicubic's taps are
        const int L = int(f.L);
        auto reflect = [L](int i) { return i < 0 ? -i : (i >= L ? 2 * (L - 1) - i : i); };
        std::vector<float> pt(size_t(L - 1) * size_t(L - 1) * kPatchFloats);
        for (int ba = 0; ba < L - 1; ++ba)
            for (int bb = 0; bb < L - 1; ++bb) {
                float* o = pt.data() + (size_t(ba) * size_t(L - 1) + size_t(bb)) * kPatchFloats;
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j)
                        for (int c = 0; c < 3; ++c)
                            o[3 * (4 * i + j) + c] =
                                f.table32[3 * (size_t(reflect(ba - 1 + i)) * size_t(L) + size_t(reflect(bb - 1 + j))) + c];
            }
        upload(pool, s, p.dev.patches, pt.data(), pt.size() * sizeof(float));
    }
    std::vector<float> c(8 * size_t(f.K));
    std::memcpy(c.data(), f.cx.data(), f.K * sizeof(float));
    std::memcpy(c.data() + f.K, f.cinv.data(), f.K * sizeof(float));
    std::memcpy(c.data() + 2 * f.K, f.cy.data(), 3 * f.K * sizeof(float));
    std::memcpy(c.data() + 5 * f.K, f.cy0.data(), 3 * f.K * sizeof(float));
    upload(pool, s, p.dev.curves, c.data(), c.size() * sizeof(float));
    if (f.grain && f.grain->K) {
        upload(pool, s, p.dev.gaxis, f.grain->axis.data(), f.grain->axis.size() * sizeof(float));
        upload(pool, s, p.dev.ginv, f.grain->inv.data(), f.grain->inv.size() * sizeof(float));
        upload(pool, s, p.dev.glayers, f.grain->layers.data(), f.grain->layers.size() * sizeof(float));
    }
    const PrintSetup& pr = *p.print;
    if (!pr.paper_tab.empty()) upload(pool, s, p.dev.paper, pr.paper_tab.data(), pr.paper_tab.size() * sizeof(float));
    upload(pool, s, p.dev.cmax, pr.cam->cmax32.data(), pr.cam->cmax32.size() * sizeof(float));
    if (pr.edr) upload(pool, s, p.dev.edr, pr.edr_tab.data(), pr.edr_tab.size() * sizeof(float));
    cuda_check(cudaStreamSynchronize(s), "table upload");
}

// ---- timing -------------------------------------------------------------------------------------

void Timer::begin(const char* name, cudaStream_t s) {
    Mark m{name, nullptr, nullptr};
    cudaEventCreate(&m.a);
    cudaEventCreate(&m.b);
    cudaEventRecord(m.a, s);
    marks.push_back(m);
}
void Timer::end(cudaStream_t s) { cudaEventRecord(marks.back().b, s); }
void Timer::before(const char* kernel, cudaStream_t s) {
    Mark m{kernel, nullptr, nullptr};
    cudaEventCreate(&m.a);
    cudaEventCreate(&m.b);
    cudaEventRecord(m.a, s);
    kernels.push_back(m);
}
void Timer::after(cudaStream_t s) { cudaEventRecord(kernels.back().b, s); }
void Timer::reset() {
    for (std::vector<Mark>* v : {&marks, &kernels}) {
        for (Mark& m : *v) {
            cudaEventDestroy(m.a);
            cudaEventDestroy(m.b);
        }
        v->clear();
    }
}
Timer::~Timer() { reset(); }

namespace {
struct Stage {
    RenderCtx& ctx;
    Stage(RenderCtx& c, const char* name) : ctx(c) {
        if (ctx.timer) ctx.timer->begin(name, ctx.stream);
    }
    ~Stage() {
        if (ctx.timer) ctx.timer->end(ctx.stream);
    }
};

// ---- the blur machinery (reference src/fx/gaussian.cpp:167-273) ----------------------------------

struct Fuse {
    int mode = ACC_NONE;
    const Plane* acc = nullptr;
    Vec3 weight{1.0, 1.0, 1.0};
};

bool same(const Plane& a, const Plane& b) { return a.data() == b.data(); }

// The kernels' direct index into an ascending axis (AxisGrid): g(v) = clamp(int((v - x0) s), 0, K - 2),
// the same binary32 operations as on the device. The grid is switched on only when, for every interval
// [x[j], x[j+1]), g stays within one of j at both ends (g rises with v, so then everywhere in between).
int grid_guess(float v, float x0, float s, uint32_t K) {
    const float t = (v - x0) * s;
    const int g = t >= float(K) ? int(K) : (t > 0.0f ? int(t) : 0);
    return std::min(std::max(g, 0), int(K) - 2);
}

AxisGrid axis_grid(const float* x, uint32_t K, uint32_t stride) {
    AxisGrid a{};
    if (K < 3) return a;
    for (uint32_t j = 0; j + 1 < K; ++j)
        if (!(x[size_t(j + 1) * stride] > x[size_t(j) * stride])) return a;
    const float x0 = x[0], xl = x[size_t(K - 1) * stride];
    const float s = f32(double(K - 1) / (double(xl) - double(x0)));
    if (!std::isfinite(s) || !(s > 0.0f)) return a;
    for (uint32_t j = 0; j + 1 < K; ++j) {
        const float lo = x[size_t(j) * stride];
        const float hi = std::nextafter(x[size_t(j + 1) * stride], -INFINITY);
        if (grid_guess(lo, x0, s, K) < int(j) - 1 || grid_guess(hi, x0, s, K) > int(j) + 1) return a;
    }
    a.x0 = x0;
    a.s = s;
    a.active = 1;
    return a;
}

// The print kernel's form of a spectral integral R_k = sum_l 10^-D(l) wt_k(l), D(l) = sum_c d_c eps_c(l)
// + beta(l) (reference kernels/print.metal:165-189): R_k = sum_l 2^(sum_c d_c e_c(l)) w_k(l) with
// e = -log2(10) eps and w_k = wt_k 10^-beta, each formed in binary64 from the binary32 tables and rounded
// once, and held twice for the packed two-pixel arithmetic.
SpectralPairs spectral_pairs(const SpectralTables& t) {
    constexpr double kNegLog2Of10 = -3.32192809488736234787;
    SpectralPairs o{};
    for (int i = 0; i < 3 * SPKB_NL; ++i) {
        const float e = f32(double(t.eps[i]) * kNegLog2Of10);
        const float w = f32(double(t.wt[i]) * std::pow(10.0, -double(t.beta[i / 3])));
        o.e[i] = F32Pair{e, e};
        o.w[i] = F32Pair{w, w};
    }
    return o;
}

FirTaps fir_taps(const Vec3& sigma, const bool iir[3]) {
    FirTaps t{};
    int r = 0;
    for (int c = 0; c < 3; ++c)
        if (!iir[c] && sigma[c] > 0.0) r = std::max(r, fir_radius(sigma[c]));
    t.r = r;
    for (int c = 0; c < 3; ++c) {
        if (iir[c] || !(sigma[c] > 0.0)) {
            t.taps[c][r] = 1.0f;
            continue;
        }
        const std::vector<double> k = gaussian_kernel(sigma[c], 3.0);
        const int rc = int(k.size() / 2);
        for (int i = -rc; i <= rc; ++i) t.taps[c][r + i] = f32(k[size_t(i + rc)]);
    }
    return t;
}

IirCoefs iir_coefs(const Vec3& sigma, const bool iir[3]) {
    IirCoefs a{};
    for (int c = 0; c < 3; ++c) {
        if (!iir[c]) continue;
        a.mask |= 1u << c;
        const IirCoefficients k = iir_coefficients(sigma[c]);
        a.B[c] = k.B;
        a.B1[c] = k.B1;
        a.B2[c] = k.B2;
        a.B3[c] = k.B3;
    }
    return a;
}

void weights(const Vec3& w, float out[3]) {
    for (int c = 0; c < 3; ++c) out[c] = f32(w[c]);
}

bool uniform_taps(const FirTaps& t) {
    for (int k = 0; k <= 2 * t.r; ++k)
        if (t.taps[1][k] != t.taps[0][k] || t.taps[2][k] != t.taps[0][k]) return false;
    return true;
}

void encode_fir(RenderCtx& ctx, const Plane& in, const Plane& dst, const FirTaps& t, const Fuse& fuse) {
    if (fuse.mode == ACC_NONE && uniform_taps(t) && dev::fir_tile_fits(in.w, in.h, t.r)) {
        // both passes in one tiled kernel (out of place; an in-place blur goes through a fresh plane)
        if (!same(in, dst)) {
            dev::fir_tile(in.data(), dst.data(), in.w, in.h, t.r, t.taps[0], ctx.stream);
            return;
        }
        Plane tmp = make_plane(ctx.pool, in.w, in.h);
        dev::fir_tile(in.data(), tmp.data(), in.w, in.h, t.r, t.taps[0], ctx.stream);
        dev::copy(tmp.data(), dst.data(), dst.pixels(), ctx.stream);
        return;
    }
    Plane tmp = make_plane(ctx.pool, in.w, in.h);
    dev::fir_v(in.data(), tmp.data(), in.w, in.h, t, ctx.stream);
    float w[3];
    weights(fuse.weight, w);
    const Plane& acc = (fuse.mode == ACC_PLANE && fuse.acc) ? *fuse.acc : dst;
    dev::fir_h(tmp.data(), dst.data(), acc.data(), in.w, in.h, t, fuse.mode, w, ctx.stream);
}

void encode_iir(RenderCtx& ctx, const Plane& in, const Plane& dst, const IirCoefs& c, const Fuse& fuse) {
    Plane tmp = make_plane(ctx.pool, in.w, in.h);
    dev::iir_h(in.data(), tmp.data(), in.w, in.h, c, ctx.stream);
    float w[3];
    weights(fuse.weight, w);
    const Plane& acc = (fuse.mode == ACC_PLANE && fuse.acc) ? *fuse.acc : dst;
    dev::iir_v(tmp.data(), dst.data(), acc.data(), in.w, in.h, c, fuse.mode, w, ctx.stream);
}

void lincomb(RenderCtx& ctx, const Vec3& a, const Plane& x, const Vec3& b, const Plane* y, const Plane& out) {
    float fa[3], fb[3];
    weights(a, fa);
    weights(b, fb);
    dev::lincomb(x.data(), y ? y->data() : nullptr, out.data(), x.pixels(), fa, fb, ctx.stream);
}

void encode_blur(RenderCtx& ctx, const Plane& in, const Plane& dst, const Vec3& sigma, const Fuse& fuse) {
    bool iir[3];
    int n_iir = 0;
    for (int c = 0; c < 3; ++c) {
        iir[c] = blur_branch(sigma[c]) == Branch::Iir;
        n_iir += iir[c];
    }
    const FirTaps fa = fir_taps(sigma, iir);
    if (n_iir == 0) {
        if (fuse.mode == ACC_NONE && fa.r == 0) {
            if (!same(in, dst)) dev::copy(in.data(), dst.data(), in.pixels(), ctx.stream);
            return;
        }
        encode_fir(ctx, in, dst, fa, fuse);
        return;
    }
    const IirCoefs ia = iir_coefs(sigma, iir);
    if (n_iir == 3) {
        encode_iir(ctx, in, dst, ia, fuse);
        return;
    }
    if (fuse.mode != ACC_NONE) {
        Plane t = make_plane(ctx.pool, in.w, in.h);
        encode_blur(ctx, in, t, sigma, Fuse{});
        if (fuse.mode == ACC_ZERO) lincomb(ctx, fuse.weight, t, Vec3{1.0, 1.0, 1.0}, nullptr, dst);
        else lincomb(ctx, Vec3{1.0, 1.0, 1.0}, *fuse.acc, fuse.weight, &t, dst);
        return;
    }
    if (fa.r > 0) {
        Plane t = make_plane(ctx.pool, in.w, in.h);
        encode_fir(ctx, in, t, fa, Fuse{});
        encode_iir(ctx, t, dst, ia, Fuse{});
    } else {
        encode_iir(ctx, in, dst, ia, Fuse{});
    }
}

}  // namespace

int blur_branch_code(double sigma) {
    switch (blur_branch(sigma)) {
        case Branch::Identity: return BLUR_IDENTITY;
        case Branch::Fir: return BLUR_FIR;
        default: return BLUR_IIR;
    }
}

FirTaps blur_fir_taps(const double sigma[3], const bool iir[3]) {
    return fir_taps(Vec3{sigma[0], sigma[1], sigma[2]}, iir);
}

IirCoefs blur_iir_coefs(const double sigma[3], const bool iir[3]) {
    return iir_coefs(Vec3{sigma[0], sigma[1], sigma[2]}, iir);
}

namespace {
bool iir_mixture_mix(RenderCtx& ctx, const Plane& raw, const std::vector<MixtureComponent>& comps, const Vec3& a,
                     const Vec3& b, bool adjoint = false);
}  // namespace

void gaussian(RenderCtx& ctx, const Plane& in, const Plane& dst, const Vec3& sigma) {
    // every channel recursive: the block-parallel kernels as a plain one-component blur, dst := G(in)
    // (the same recurrence as the line kernels, evaluated by segments; in == dst allowed)
    if (blur_branch(sigma[0]) == Branch::Iir && blur_branch(sigma[1]) == Branch::Iir &&
        blur_branch(sigma[2]) == Branch::Iir && dev::iir_mixture_fits(in.w, in.h)) {
        const double s3[3] = {sigma[0], sigma[1], sigma[2]};
        const bool all[3] = {true, true, true};
        Plane tmp = make_plane(ctx.pool, in.w, in.h);
        if (blur_iir_block(in.data(), dst.data(), tmp.data(), in.w, in.h, s3, all, ctx.stream)) return;
    }
    encode_blur(ctx, in, dst, sigma, Fuse{});
}

void gaussian_mixture(RenderCtx& ctx, const Plane& in, const Plane& out, const std::vector<MixtureComponent>& comps) {
    if (comps.empty()) fail_internal("empty mixture");
    Plane acc = same(in, out) ? make_plane(ctx.pool, in.w, in.h) : out;
    for (size_t k = 0; k < comps.size(); ++k) {
        const MixtureComponent& m = comps[k];
        const bool ident = !(m.sigma[0] > 0.0) && !(m.sigma[1] > 0.0) && !(m.sigma[2] > 0.0);
        if (k == 0 && ident) {
            lincomb(ctx, Vec3{0.0, 0.0, 0.0}, in, m.weight, &in, acc);
            continue;
        }
        Fuse f;
        f.mode = k == 0 ? ACC_ZERO : ACC_PLANE;
        f.acc = &acc;
        f.weight = m.weight;
        encode_blur(ctx, in, acc, m.sigma, f);
    }
    if (!same(acc, out)) dev::copy(acc.data(), out.data(), acc.pixels(), ctx.stream);
}

namespace {

// M: the map of an entry state (s1, s2, s3) through L steps of the homogeneous recurrence.
void entry_map(const IirCoefficients& k, int L, double M[3][3]) {
    for (int j = 0; j < 3; ++j) {
        double s[3] = {0.0, 0.0, 0.0};
        s[j] = 1.0;
        for (int i = 0; i < L; ++i) {
            const double t = (k.B1 * s[0] + k.B2 * s[1]) + k.B3 * s[2];
            s[2] = s[1];
            s[1] = s[0];
            s[0] = t;
        }
        for (int r = 0; r < 3; ++r) M[r][j] = s[r];
    }
}

// active: the channels that blur (null: all three); the others pass through
void fill_launch(dev::IirLaunch& q, const std::vector<MixtureComponent>& comps, int L, const bool* active = nullptr) {
    q.seg_len = L;
    for (size_t c = 0; c < comps.size(); ++c)
        for (int ch = 0; ch < 3; ++ch) {
            dev::IirChannel& d = q.ch[3 * c + ch];
            if (active && !active[ch]) {
                d = dev::IirChannel{};
                continue;
            }
            const IirCoefficients k = iir_coefficients(comps[c].sigma[ch]);
            d.B = k.B;
            d.B1 = k.B1;
            d.B2 = k.B2;
            d.B3 = k.B3;
            // M^(2^p), the map through L 2^p steps: the map through L steps, then squared (7 products of
            // 3 x 3 matrices instead of 381 L steps of the recurrence on the host before every launch)
            entry_map(k, L, d.Mp[0]);
            for (int p = 1; p < dev::kIirScanSteps; ++p)
                for (int r = 0; r < 3; ++r)
                    for (int c2 = 0; c2 < 3; ++c2)
                        d.Mp[p][r][c2] = (d.Mp[p - 1][r][0] * d.Mp[p - 1][0][c2] + d.Mp[p - 1][r][1] * d.Mp[p - 1][1][c2]) +
                                         d.Mp[p - 1][r][2] * d.Mp[p - 1][2][c2];
            d.active = 1;
        }
}

// raw := a raw + b M(raw) with the block-parallel recursive kernels, when every channel of every
// component is on the recursive branch and the lines fit in shared memory; false otherwise.
bool iir_mixture_mix(RenderCtx& ctx, const Plane& raw, const std::vector<MixtureComponent>& comps, const Vec3& a,
                     const Vec3& b, bool adjoint) {
    if (comps.empty() || comps.size() > SPKB_MAX_COMPONENTS) return false;
    for (const MixtureComponent& m : comps)
        for (int c = 0; c < 3; ++c)
            if (blur_branch(m.sigma[c]) != Branch::Iir) return false;
    if (!dev::iir_mixture_fits(raw.w, raw.h)) return false;
    dev::IirMixture q{};
    q.ncomp = uint32_t(comps.size());
    for (size_t c = 0; c < comps.size(); ++c) weights(comps[c].weight, q.weight[c]);
    weights(a, q.mix_a);
    weights(b, q.mix_b);
    const int Lr = dev::iir_row_seg_len(raw.w);
    const int Lc = dev::iir_col_seg_len(raw.h);
    fill_launch(q.rows, comps, Lr);
    fill_launch(q.cols, comps, Lc);
    q.rows.adjoint = q.cols.adjoint = adjoint ? 1 : 0;
    std::vector<Plane> tmp;
    float* tp[SPKB_MAX_COMPONENTS] = {};
    for (size_t c = 0; c < comps.size(); ++c) {
        tmp.push_back(make_plane(ctx.pool, raw.w, raw.h));
        tp[c] = tmp.back().data();
    }
    Plane acc = comps.size() > 1 ? make_plane(ctx.pool, raw.w, raw.h) : Plane{};
    dev::iir_mixture(raw.data(), raw.data(), tp, acc ? acc.data() : nullptr, raw.w, raw.h, q, ctx.stream);
    return true;
}

}  // namespace

bool blur_iir_block(const float* src, float* dst, float* tmp, uint32_t w, uint32_t h, const double sigma[3],
                    const bool iir[3], cudaStream_t s) {
    // the kernels move whole rows and strips in 16-byte pieces from the planes' bases
    auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (!aligned(src) || !aligned(dst) || !aligned(tmp) || !dev::iir_mixture_fits(w, h)) return false;
    dev::IirMixture q{};
    q.ncomp = 1;
    q.plain = 1;
    const std::vector<MixtureComponent> one{MixtureComponent{Vec3{1.0, 1.0, 1.0}, Vec3{sigma[0], sigma[1], sigma[2]}}};
    fill_launch(q.rows, one, dev::iir_row_seg_len(w), iir);
    fill_launch(q.cols, one, dev::iir_col_seg_len(h), iir);
    float* tp[SPKB_MAX_COMPONENTS] = {tmp};
    dev::iir_mixture(src, dst, tp, nullptr, w, h, q, s);
    return true;
}

void check_supported(const ParamSet&) {
    // every field of the reference's parameter schema has its stage in this build: nothing is refused
}

namespace {

ExposeArgs expose_args(const FilmSetup& f, size_t pixels) {
    ExposeArgs a{};
    for (int i = 0; i < 9; ++i) a.a[i] = f.input_matrix_f32[size_t(i)];
    a.gain = f32(std::pow(2.0, f.params.f(P::exposure_compensation_ev)));
    a.apply_gain = a.gain != 1.0f;
    a.L = f.L;
    a.n = uint32_t(pixels);
    return a;
}

// the camera lens blur of the film side in pixels (0: none)
double film_lens_blur_px(const RenderCtx& ctx, const FilmSetup& f) {
    const double um = f.params.f(P::lens_blur_um);
    return um > 0.0 ? um / ctx.pitch_um : 0.0;
}

// the film's halation stages: the override's bounce mixture, or the film preset's plan at this pitch
HalationPlan film_halation(const RenderCtx& ctx, const FilmSetup& f, const std::optional<HalationOverride>& hov) {
    HalationPlan pl;
    if (hov) {
        pl.bounce = !hov->comps.empty();
        pl.bounce_comps = hov->comps;
        for (size_t c = 0; c < 3; ++c) {
            const double A = hov->strength[c];
            pl.mix_a[c] = 1.0 / (1.0 + A);
            pl.mix_b[c] = A / (1.0 + A);
        }
        return pl;
    }
    return halation_plan(f.halation, ctx.pitch_um);
}

// raw := a raw + b M(raw) for the scatter, then the bounce mixture
void apply_halation(RenderCtx& ctx, const HalationPlan& pl, Plane& H) {
    if (pl.scatter && !iir_mixture_mix(ctx, H, pl.scatter_comps, pl.scatter_a, pl.scatter_b)) {
        Plane m = make_plane(ctx.pool, H.w, H.h);
        gaussian_mixture(ctx, H, m, pl.scatter_comps);
        lincomb(ctx, pl.scatter_a, H, pl.scatter_b, &m, H);
    }
    if (pl.bounce && !iir_mixture_mix(ctx, H, pl.bounce_comps, pl.mix_a, pl.mix_b)) {
        Plane Hh = make_plane(ctx.pool, H.w, H.h);
        gaussian_mixture(ctx, H, Hh, pl.bounce_comps);
        lincomb(ctx, pl.mix_a, H, pl.mix_b, &Hh, H);
    }
}

struct DevelopPlan {
    DevelopArgs da{};
    bool grain = false;
    double final_blur = 0.0, amount = 1.0;
};

// the develop kernel's arguments for a frame of width w and the grain's final blur and strength
DevelopPlan develop_plan(const RenderCtx& ctx, const Pipeline& p, uint32_t w, uint32_t film_seed, float* counts_out,
                         float* lam_out = nullptr) {
    const FilmSetup& f = *p.film;
    DevelopPlan dp;
    DevelopArgs& da = dp.da;
    da.cx = p.dev.curves.as<float>();
    da.cinv = da.cx + f.K;
    da.cy = da.cx + 2 * size_t(f.K);
    da.K = f.K;
    da.cgrid = axis_grid(f.cx.data(), f.K, 1);
    da.width = w;
    da.counts_out = counts_out;
    da.lam_out = lam_out;
    const GrainSetup* g = f.grain.get();
    dp.grain = g && g->active && g->amount > 0.0;
    if (!dp.grain) return dp;
    const GrainConstants kc = grain_constants(*g, ctx.pitch_um);
    if (kc.sublayers && (kc.dye || kc.micro))
        fail_user("grain dye clouds or micro-structure (pixel pitch below about 2 um) are outside this B200 build's render path");
    dp.final_blur = kc.final_blur;
    dp.amount = g->amount;
    da.grain = 1;
    da.seed = film_seed;
    da.positive = g->positive ? 1u : 0u;
    da.n_sub = 1;
    da.inv_n_sub = f32(1.0);
    for (size_t c = 0; c < 3; ++c) {
        da.uniformity[c] = f32(c == 1 ? 0.99 : 0.97);
        da.dmin_c[c] = f32(kGrainDmin[c]);
    }
    for (size_t l = 0; l < 3; ++l)
        for (size_t c = 0; c < 3; ++c) {
            da.dmin_l[l * 3 + c] = f32(kc.dmin_l[l][c]);
            da.sat_d[l * 3 + c] = f32(kc.sat_d[l][c]);
            da.count[l * 3 + c] = f32(kc.count[l][c]);
            da.unit[l * 3 + c] = da.sat_d[l * 3 + c] / da.count[l * 3 + c];
        }
    if (g->sublayers) {
        da.mode = 0;  // SUM
        da.shift = 1;
        da.gK = g->K;
        da.axis = p.dev.gaxis.as<float>();
        da.ginv = p.dev.ginv.as<float>();
        da.layers = p.dev.glayers.as<float>();
        for (uint32_t c = 0; c < 3; ++c) da.ggrid[c] = axis_grid(g->axis.data() + c, g->K, 3);
    } else {
        da.mode = 2;  // SIMPLE
    }
    return dp;
}

}  // namespace

std::vector<MixtureComponent> dir_diffusion_components(double pitch_um) {
    constexpr double kCoreUm = 20.0, kTailUm = 200.0, kTailWeight = 0.06;
    std::vector<MixtureComponent> comps;
    MixtureComponent core;
    const double s = kCoreUm / pitch_um;
    for (int c = 0; c < 3; ++c) {
        core.weight[c] = 1.0 - kTailWeight;
        core.sigma[c] = s;
    }
    comps.push_back(core);
    const double lam = kTailUm / pitch_um;
    for (const MixtureComponent& m : exponential_surrogate(Vec3{kTailWeight, kTailWeight, kTailWeight}, Vec3{lam, lam, lam}))
        comps.push_back(m);
    return comps;
}

namespace {
// DIR couplers (reference src/film/develop.cpp:203-226): the correction chi from the first development of
// the exposure H, blurred by the diffusion mixture; the develop then reads the pre-inverted curve y0 at the
// log exposure minus chi (da.cy, da.chi set here).
Plane dir_couplers(RenderCtx& ctx, const Pipeline& p, const Plane& H, DevelopArgs& da) {
    const FilmSetup& f = *p.film;
    if (!(ctx.pitch_um > 0.0)) fail_internal("DIR couplers without a pixel pitch");
    CouplerArgs q{};
    q.cx = da.cx;
    q.cinv = da.cinv;
    q.cy = da.cy;
    q.K = da.K;
    q.cgrid = da.cgrid;
    q.positive = f.positive ? 1u : 0u;
    for (int i = 0; i < 9; ++i) q.m[i] = f.coupler_m_f32[size_t(i)];
    for (int c = 0; c < 3; ++c) q.dmax[c] = f.dmax_f32[size_t(c)];
    q.n = uint32_t(H.pixels());
    Plane chi = make_plane(ctx.pool, H.w, H.h);
    dev::coupler_source(H.data(), chi.data(), q, ctx.stream);
    // the diffusion: the FIR components (the 20 um core below 60 um pitch) into a side plane, the recursive
    // ones (the tail's surrogate) in one block-parallel mixture launch pair in place, then their sum
    const std::vector<MixtureComponent> comps = dir_diffusion_components(ctx.pitch_um);
    std::vector<MixtureComponent> fir, iir;
    for (const MixtureComponent& m : comps) {
        bool rec = true;
        for (int c = 0; c < 3; ++c) rec = rec && blur_branch(m.sigma[c]) == Branch::Iir;
        (rec ? iir : fir).push_back(m);
    }
    if (iir.empty() || fir.size() > 1 || !dev::iir_mixture_fits(chi.w, chi.h)) {
        gaussian_mixture(ctx, chi, chi, comps);
    } else {
        Plane core;
        if (!fir.empty()) {
            core = make_plane(ctx.pool, chi.w, chi.h);
            Fuse f;
            f.mode = ACC_ZERO;
            f.acc = &core;
            f.weight = fir[0].weight;
            encode_blur(ctx, chi, core, fir[0].sigma, f);
        }
        if (!iir_mixture_mix(ctx, chi, iir, Vec3{0.0, 0.0, 0.0}, Vec3{1.0, 1.0, 1.0}))
            fail_internal("DIR diffusion: the recursive mixture was refused");
        if (core) lincomb(ctx, Vec3{1.0, 1.0, 1.0}, core, Vec3{1.0, 1.0, 1.0}, &chi, chi);
    }
    da.cy = da.cx + 5 * size_t(f.K);
    da.chi = chi.data();
    return chi;
}
}  // namespace

bool headroom_applies(const HalationParams& h) {
    return h.active && h.back_reflection && h.headroom_ev > 0.0 && h.amount > 0.0;
}

namespace {
// The highlight boost (reference src/film/develop.cpp:32-62): values above x0 = min(0.184 2^4, M) lifted
// by k M (exp(z) - z - 1), z = a (v - x0) / M, with M the frame maximum (read back: the constants are
// binary64 functions of it) and k from boost_ev; M = 0 scales the frame by 0.
void run_boost(RenderCtx& ctx, const Plane& H, double beta_ev) {
    DevBuffer mx = ctx.pool.acquire(16);
    uint32_t* ord = mx.as<uint32_t>();
    float* val = reinterpret_cast<float*>(ord + 1);
    dev::plane_max(H.data(), 3 * H.pixels(), ord, ctx.stream);
    dev::plane_max_value(ord, val, ctx.stream);
    float M = 0.0f;
    cuda_check(cudaMemcpyAsync(&M, val, sizeof M, cudaMemcpyDeviceToHost, ctx.stream), "frame maximum");
    cuda_check(cudaStreamSynchronize(ctx.stream), "frame maximum");
    if (M == 0.0f) {
        const float zero[3] = {0.0f, 0.0f, 0.0f};
        dev::lincomb(H.data(), nullptr, H.data(), H.pixels(), zero, zero, ctx.stream);
        return;
    }
    const double Md = double(M);
    const double x0 = std::min(std::max(0.184 * std::pow(2.0, 4.0), 0.0), Md);
    if (x0 == Md) return;
    const double a = std::pow(28.0, 1.0 - 0.3);
    const double q = a * (1.0 - x0 / Md);
    const double den = std::exp(q) - q - 1.0;
    if (!(den > 0.0)) fail_gpu("highlight boost: the frame maximum leaves no range to lift (den <= 0)");
    const double k = (std::pow(2.0, beta_ev) - 1.0) / den;
    dev::boost(H.data(), 3 * H.pixels(), f32(x0), f32(1.0 / Md), f32(a), f32(k * Md), ctx.stream);
}
}  // namespace

Plane develop(RenderCtx& ctx, const Pipeline& p, const Plane& tier_source, uint32_t film_seed,
              const std::optional<HalationOverride>& hov, float* counts_out, float* lam_out) {
    const FilmSetup& f = *p.film;
    Plane source = tier_source;
    if (f.decode) ctx.node("preprocess.decode");
    if (!geometry_identity(f.params)) ctx.node("preprocess.geometry");
    if (f.decode || !geometry_identity(f.params)) {
        Stage st(ctx, "prepare");
        source = prepare_source(ctx.pool, ctx.stream, tier_source, f.params, f.decode, uint32_t(f.input_space.cctf));
    }
    const uint32_t w = source.w, h = source.h;
    Plane H = make_plane(ctx.pool, w, h);
    if (f.params.b(P::auto_exposure)) ctx.node("filming.auto_exposure");
    ctx.node("filming.upsample");
    ctx.node("filming.exposure_compensation");
    {
        Stage st(ctx, "expose");
        ExposeArgs ea = expose_args(f, source.pixels());
        if (f.params.b(P::auto_exposure) && ctx.ae_ev) {
            ea.ae_gain = f32(std::pow(2.0, *ctx.ae_ev));
            ea.apply_ae = 1;
        }
        dev::expose(source.data(), H.data(), p.dev.table.as<float>(), p.dev.patches.as<float>(), ea, ctx.stream);
    }
    if (const double bev = f.params.f(P::halation_boost_ev); bev != 0.0) {
        ctx.node("filming.boost");
        Stage st(ctx, "boost");
        run_boost(ctx, H, bev);
    }
    if (headroom_applies(f.halation)) {
        // the back-reflection halation's highlight headroom, its clip the frame maximum kept on the device
        ctx.node("filming.headroom");
        Stage st(ctx, "headroom");
        DevBuffer mx = ctx.pool.acquire(16);
        dev::plane_max(H.data(), 3 * H.pixels(), mx.as<uint32_t>(), ctx.stream);
        dev::headroom(H.data(), uint32_t(H.pixels()), mx.as<uint32_t>(), f32(f.halation.headroom_ev), ctx.stream);
    }
    if (f.params.f(P::lens_blur_um) > 0.0) ctx.node("filming.lens_blur");
    if (const double s = film_lens_blur_px(ctx, f); s > 0.0) {
        Stage st(ctx, "lens_blur");
        Plane Hb = make_plane(ctx.pool, w, h);
        gaussian(ctx, H, Hb, Vec3{s, s, s});
        H = std::move(Hb);
    }
    {
        const HalationPlan pl = film_halation(ctx, f, hov);
        if (pl.scatter || pl.bounce) {
            ctx.node("filming.halation");
            Stage st(ctx, "halation");
            apply_halation(ctx, pl, H);
        }
    }
    DevelopPlan dp = develop_plan(ctx, p, w, film_seed, counts_out, lam_out);
    ctx.node("filming.log");  // log, curves, couplers and grain are fused into the develop launches
    ctx.node("filming.curves");
    if (f.couplers) ctx.node("filming.couplers");
    if (f.grain) ctx.node("filming.grain");
    Plane chi;
    if (f.couplers) {
        Stage st(ctx, "couplers");
        chi = dir_couplers(ctx, p, H, dp.da);
    }
    const DevelopArgs& da = dp.da;
    Plane neg = make_plane(ctx.pool, w, h);
    if (!dp.grain) {
        Stage st(ctx, "develop");
        dev::develop(H.data(), neg.data(), da, w, h, ctx.stream);
        return neg;
    }
    Plane G = make_plane(ctx.pool, w, h);
    {
        Stage st(ctx, "develop");
        dev::develop(H.data(), G.data(), da, w, h, ctx.stream);
    }
    if (dp.final_blur > 0.0) {
        Stage st(ctx, "grain_blur");
        const double s = dp.final_blur;
        if (dp.amount == 1.0) {  // the blurred grain is the negative
            gaussian(ctx, G, neg, Vec3{s, s, s});
            return neg;
        }
        Plane Gb = make_plane(ctx.pool, w, h);
        gaussian(ctx, G, Gb, Vec3{s, s, s});
        G = std::move(Gb);
    }
    {
        Stage st(ctx, "grain_mix");
        if (dp.amount == 1.0) {
            dev::copy(G.data(), neg.data(), G.pixels(), ctx.stream);
        } else {
            DevelopArgs dd = da;
            dd.grain = 0;
            dev::develop(H.data(), neg.data(), dd, w, h, ctx.stream);
            const double k = dp.amount;
            lincomb(ctx, Vec3{1.0 - k, 1.0 - k, 1.0 - k}, neg, Vec3{k, k, k}, &G, neg);
        }
    }
    return neg;
}

namespace {
uint16_t bf16_rn(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}
float bf16_value(uint16_t h) {
    const uint32_t u = uint32_t(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// One integral of the spectral-mode kernel from its binary64 tables at the resources' 81 wavelengths
// (eps [l][c], beta [l], wt [l][k]) and their binary32 narrowings t32. At 81 wavelengths the binary32
// values are the print kernel's (spectral_pairs); at 1 nm the binary64 tables are interpolated linearly and
// a bin's weight is a fifth of a 5 nm bin's, so that the sum approximates the same integral.
void fill_spectral_pass(SpectralTablesN& t, uint32_t pass, const double* eps64, const double* beta64,
                        const double* wt64, const SpectralTables& t32) {
    constexpr double kNegLog2Of10 = -3.32192809488736234787;
    const uint32_t nl = t.nl, np = t.nl_pad;
    const double step = double(SPKB_NL - 1) / double(nl - 1);
    for (uint32_t l = 0; l < nl; ++l) {
        double eps[3], wt[3], beta;
        float e32[3], w32[3];
        if (nl == SPKB_NL) {
            beta = beta64[l];
            for (int c = 0; c < 3; ++c) {
                eps[c] = eps64[3 * l + c];
                wt[c] = wt64[3 * l + c];
                e32[c] = f32(double(t32.eps[3 * l + c]) * kNegLog2Of10);
                w32[c] = f32(double(t32.wt[3 * l + c]) * std::pow(10.0, -double(t32.beta[l])));
            }
        } else {
            const double x = double(l) * step;
            const uint32_t i = std::min(uint32_t(x), uint32_t(SPKB_NL - 2));
            const double f = x - double(i);
            beta = (1.0 - f) * beta64[i] + f * beta64[i + 1];
            for (int c = 0; c < 3; ++c) {
                eps[c] = (1.0 - f) * eps64[3 * i + c] + f * eps64[3 * (i + 1) + c];
                wt[c] = ((1.0 - f) * wt64[3 * i + c] + f * wt64[3 * (i + 1) + c]) * step;
                e32[c] = f32(eps[c] * kNegLog2Of10);
                w32[c] = f32(wt[c] * std::pow(10.0, -beta));
            }
        }
        for (uint32_t c = 0; c < 3; ++c) {
            t.e64[pass][l][c] = eps[c] * kNegLog2Of10;
            t.w64[pass][l][c] = wt[c] * std::pow(10.0, -beta);
            t.e_pairs[pass][l / 2][2 * c + (l & 1)] = e32[c];
            t.w[pass][l][c] = w32[c];
            const uint16_t hi = bf16_rn(w32[c]);
            const uint16_t lo = bf16_rn(w32[c] - bf16_value(hi));
            auto at = [&](uint32_t n, uint32_t bytes) {  // element index of (n, l) in the B tile
                const uint32_t b = ((n / 8) * (np * bytes / 16) + (l * bytes) / 16) * 128 + (n % 8) * 16 + (l * bytes) % 16;
                return b / bytes;
            };
            t.b_bf16[pass][at(c, 2)] = hi;
            t.b_bf16[pass][at(3 + c, 2)] = lo;
            t.b_tf32[pass][at(c, 4)] = w32[c];
        }
    }
}
}  // namespace

void spectral_tables_n(const PrintSetup& s, const PrintRun& r, uint32_t bins, SpectralTablesN& t) {
    if (bins != SPKB_NL && bins != 401) fail_invalid("spectral print: 81 or 401 wavelengths");
    std::memset(&t, 0, sizeof t);
    t.nl = bins;
    t.nl_pad = (bins + 31) / 32 * 32;
    fill_spectral_pass(t, 0, r.eps_n.data(), r.beta_n.data(), r.w_n.data(), r.enl32);
    fill_spectral_pass(t, 1, s.scan_eps.data(), s.scan_beta.data(), s.scan_wt.data(), s.scan32);
}

PrintArgs print_args(const Pipeline& p, const LiveParams& live, uint32_t pixels) {
    const PrintSetup& s = *p.print;
    const PrintRun r = compute_run(s, live);
    PrintArgs a{};
    a.enl = spectral_pairs(r.enl32);
    a.scan = spectral_pairs(s.scan32);
    for (int c = 0; c < 3; ++c) {
        a.g[c] = f32(r.g[c]);
        a.o[c] = f32(r.o[c]);
    }
    a.k_gain = r.k_gain;
    a.printed = s.scanned ? 0 : 1;
    a.paper = p.dev.paper.as<float>();
    a.paper_K = s.paper_K;
    if (!s.paper_tab.empty()) a.paper_grid = axis_grid(s.paper_tab.data(), s.paper_K, 1);
    std::memcpy(a.to_rgb, s.to_rgb, sizeof a.to_rgb);
    a.cam = s.cam_args;
    a.cmax = p.dev.cmax.as<float>();
    a.n = pixels;
    for (int c = 0; c < 3; ++c) a.glare_tint[c] = f32(p.print->glare_tint[size_t(c)]);
    a.levels = r.levels ? 1 : 0;
    a.levels_m = f32(r.m);
    a.levels_q = f32(r.q);
    return a;
}

namespace {
EncodeArgs encode_args(const Pipeline& p, uint32_t stride_px) {
    const PrintSetup& s = *p.print;
    EncodeArgs e{};
    std::memcpy(e.m_nid, s.m_nid, sizeof e.m_nid);
    e.cctf_active = s.cctf ? 1 : 0;
    e.cctf_mode = s.cctf_mode;
    e.stride = stride_px;
    if (s.edr && !s.scanned) {  // the EDR tone map of a printed frame (reference src/print/run.cpp:177-180)
        e.edr = 1;
        e.edr_n = uint32_t(s.edr_tab.size());
        for (int c = 0; c < 3; ++c) e.edr_r_y[c] = f32(s.out_cs.rgb_to_xyz[size_t(3 + c)]);
        e.edr_lo = f32(s.edr_lo);
        e.edr_span = f32(s.edr_hi - s.edr_lo);
        e.edr_toe = f32(s.edr_toe);
        e.edr_shoulder = f32(s.edr_shoulder);
        e.edr_tab = p.dev.edr.as<float>();
    }
    return e;
}
}  // namespace

bool scan_args(const Pipeline& p, double rho_tier, uint32_t w, uint32_t h, uint32_t stride_px, ScanArgs& sa) {
    const PrintSetup& s = *p.print;
    const double sb = s.scanner_lens_blur_px;
    const double su = s.unsharp_sigma_full * rho_tier;
    const double am = s.unsharp_amount;
    const bool unsharp = su > 0.0 && am > 0.0;
    const Branch bb = blur_branch(sb), bu = unsharp ? blur_branch(su) : Branch::Identity;
    if (bb == Branch::Iir || bu == Branch::Iir) return false;
    const bool no_iir[3] = {false, false, false};
    const FirTaps t1 = fir_taps(Vec3{sb, sb, sb}, no_iir);
    const FirTaps t2 = fir_taps(Vec3{su, su, su}, no_iir);
    sa = ScanArgs{};
    sa.r1 = t1.r;
    std::memcpy(sa.t1, t1.taps[0], sizeof sa.t1);
    sa.r2 = unsharp ? t2.r : 0;
    if (unsharp) std::memcpy(sa.t2, t2.taps[0], sizeof sa.t2);
    if (sa.r1 == 0) sa.t1[0] = 1.0f;
    if (sa.r2 == 0) sa.t2[0] = 1.0f;
    if (!dev::scan_encode_fits(w, h, sa.r1, sa.r2)) return false;
    sa.e = encode_args(p, stride_px);
    sa.e.unsharp = unsharp ? 1 : 0;
    sa.e.lincomb_a = f32(1.0 + am);
    sa.e.lincomb_b = f32(-am);
    return true;
}

Plane glare_plane(RenderCtx& ctx, const Pipeline& p, uint32_t w, uint32_t h) {
    const PrintSetup& s = *p.print;
    if (s.scanned || !s.glare_draws()) return {};
    const double pp = s.glare_percent * s.glare_amount;
    Plane f = make_plane(ctx.pool, w, h);
    dev::glare_field(f.data(), w * h, f32(pp), f32(s.glare_roughness * pp), ctx.print_seed, ctx.stream);
    if (!(s.glare_blur_full > 0.0)) return f;
    // blurred out of place: the tiled FIR then writes its result once, with no copy back
    const double sg = s.glare_blur_full * ctx.rho_tier * std::sqrt(std::max(s.glare_amount, 0.0));
    Plane blurred = make_plane(ctx.pool, w, h);
    gaussian(ctx, f, blurred, Vec3{sg, sg, sg});
    return blurred;
}

namespace {
// negative -> linear output RGB by the binary32 print kernel, or by the spectral-mode kernel when the
// context asks for one (its tables and arguments uploaded for the call, its wait status read back)
void print_stage(RenderCtx& ctx, const Pipeline& p, const LiveParams& live, const Plane& negative, const Plane& rgb,
                 const float* glare) {
    const uint32_t n = uint32_t(negative.pixels());
    PrintArgs a = print_args(p, live, n);
    a.glare = glare;
    if (ctx.print_mode < 0) {
        dev::print(negative.data(), rgb.data(), a, ctx.stream);
        return;
    }
    auto tabs = std::make_unique<SpectralTablesN>();
    spectral_tables_n(*p.print, compute_run(*p.print, live), ctx.print_bins, *tabs);
    if (!dev::print_spectral_supported(tabs->nl_pad)) fail_invalid("spectral print: 81 or 401 wavelengths");
    DevBuffer tab_d = ctx.pool.acquire(sizeof(SpectralTablesN));
    DevBuffer err_d = ctx.pool.acquire(16);
    // a pageable source: the copy has read it when the call returns
    cuda_check(cudaMemcpyAsync(tab_d.ptr(), tabs.get(), sizeof(SpectralTablesN), cudaMemcpyHostToDevice, ctx.stream),
               "spectral tables");
    cuda_check(cudaMemsetAsync(err_d.ptr(), 0, 16, ctx.stream), "print status");
    dev::print_spectral(a, *tabs, tab_d.as<SpectralTablesN>(), ctx.print_mode, negative.data(), rgb.data(), n,
                        ctx.contraction_out, err_d.as<uint32_t>(), ctx.stream);
    cuda_check(cudaGetLastError(), "print_spectral");
    uint32_t err = 0;
    cuda_check(cudaMemcpyAsync(&err, err_d.ptr(), 4, cudaMemcpyDeviceToHost, ctx.stream), "print status");
    cuda_check(cudaStreamSynchronize(ctx.stream), "print");
    if (err) fail_gpu("print: a tensor-core wait gave up");
}
}  // namespace

namespace {
constexpr uint32_t kBandRows = 8 * dev::scan_tile_rows();

// The print and the tiled scanner in row bands, each band's RGBA16 rows copied to the host on the copy
// stream while the next band's kernels run. Band b's scanner reads the print output up to kernel radius
// r1 + r2 rows past its last row, so the print runs that far ahead; the print is per pixel and the scanner
// per tile, so the bands write what the whole-frame launches write.
void print_scan_banded(RenderCtx& ctx, const Pipeline& p, const LiveParams& live, const Plane& negative,
                       const Plane& rgb, OutputImage* img, const ScanArgs& sa, const float* glare) {
    const uint32_t w = negative.w, h = negative.h;
    const uint32_t halo = uint32_t(sa.r1 + sa.r2);
    const uint32_t nb = (h + kBandRows - 1) / kBandRows;
    std::vector<cudaEvent_t>& ev = *ctx.band_events;
    while (ev.size() < nb + 1) {
        cudaEvent_t e = nullptr;
        cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "band event");
        ev.push_back(e);
    }
    PrintArgs a = print_args(p, live, 0);
    const size_t row_bytes = size_t(img->stride_px) * 4 * sizeof(uint16_t);
    uint32_t printed = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t r0 = b * kBandRows, r1 = std::min(h, r0 + kBandRows);
        const uint32_t need = std::min(h, r1 + halo);
        if (need > printed) {
            a.n = (need - printed) * w;
            a.glare = glare ? glare + size_t(printed) * w * 3 : nullptr;
            dev::print(negative.data() + size_t(printed) * w * 3, rgb.data() + size_t(printed) * w * 3, a, ctx.stream);
            printed = need;
        }
        dev::scan_encode_rows(rgb.data(), img->dev, w, h, r0, r1, sa, ctx.stream);
        cuda_check(cudaEventRecord(ev[b], ctx.stream), "band event");
        cuda_check(cudaStreamWaitEvent(ctx.copy_stream, ev[b], 0), "band event");
        cuda_check(cudaMemcpyAsync(reinterpret_cast<unsigned char*>(img->host) + size_t(r0) * row_bytes,
                                   reinterpret_cast<const unsigned char*>(img->dev) + size_t(r0) * row_bytes,
                                   size_t(r1 - r0) * row_bytes, cudaMemcpyDeviceToHost, ctx.copy_stream),
                   "result copy");
    }
    cuda_check(cudaEventRecord(ev[nb], ctx.copy_stream), "band event");
    cuda_check(cudaStreamWaitEvent(ctx.stream, ev[nb], 0), "band event");
}
}  // namespace

uint32_t film_node_count(const FilmSetup& f) {
    uint32_t n = 4;  // upsample, exposure compensation, log and curves
    if (f.decode) ++n;
    if (!geometry_identity(f.params)) ++n;
    if (f.params.b(P::auto_exposure)) ++n;
    if (f.params.f(P::halation_boost_ev) != 0.0) ++n;
    if (headroom_applies(f.halation)) ++n;
    if (f.params.f(P::lens_blur_um) > 0.0) ++n;
    if (f.halation.active) ++n;
    if (f.couplers) ++n;
    if (f.grain) ++n;
    return n;
}

uint32_t print_node_count(const PrintSetup& s) {
    const bool printed = !s.scanned;
    uint32_t n = 5;  // scan, to_rgb, gamut, scanner and encode (the desktop variant keeps the scanner)
    if (printed) n += 3;
    if (s.levels_active()) ++n;
    if (printed && s.glare_draws()) ++n;
    if (printed && s.edr) ++n;
    return n;
}

namespace {
// labels before the print launch: enlarger, gain, paper, scan, levels, glare, to_rgb, gamut
void print_nodes_head(RenderCtx& ctx, const PrintSetup& s) {
    const bool printed = !s.scanned;
    if (printed) {
        ctx.node("printing.enlarger");
        ctx.node("printing.gain");
        ctx.node("printing.paper");
    }
    ctx.node("scanning.scan");
    if (s.levels_active()) ctx.node("scanning.levels");
    if (printed && s.glare_draws()) ctx.node("scanning.glare");
    ctx.node("scanning.to_rgb");
    ctx.node("scanning.gamut");
}
// labels before the scanner launch: scanner, EDR, encode
void print_nodes_tail(RenderCtx& ctx, const PrintSetup& s) {
    ctx.node("scanning.scanner");
    if (!s.scanned && s.edr) ctx.node("scanning.edr");
    ctx.node("scanning.encode");
}
}  // namespace

void print_nodes(RenderCtx& ctx, const PrintSetup& s) {
    print_nodes_head(ctx, s);
    print_nodes_tail(ctx, s);
}

bool print_scan_encode(RenderCtx& ctx, const Pipeline& p, const LiveParams& live, const Plane& negative,
                       OutputImage* img, bool to_host) {
    const PrintSetup& s = *p.print;
    print_nodes_head(ctx, s);
    const uint32_t w = negative.w, h = negative.h;
    Plane rgb = make_plane(ctx.pool, w, h);
    Plane glare;
    if (!s.scanned && s.glare_draws()) {
        Stage st(ctx, "glare");
        glare = glare_plane(ctx, p, w, h);
    }
    const float* gl = glare ? glare.data() : nullptr;
    ScanArgs sa;
    const bool tiled = scan_args(p, ctx.rho_tier, w, h, img->stride_px, sa);
    if (to_host && tiled && ctx.print_mode < 0 && ctx.copy_stream && ctx.band_events && h > kBandRows) {
        print_nodes_tail(ctx, s);
        Stage st(ctx, "print_scanner");
        print_scan_banded(ctx, p, live, negative, rgb, img, sa, gl);
        return true;
    }
    {
        Stage st(ctx, "print");
        print_stage(ctx, p, live, negative, rgb, gl);
    }
    print_nodes_tail(ctx, s);
    if (tiled) {
        // the scanner's blurs on the FIR branch: one tiled pass from the print output to RGBA16
        Stage st(ctx, "scanner");
        dev::scan_encode(rgb.data(), img->dev, w, h, sa, ctx.stream);
        return false;
    }
    EncodeArgs e = encode_args(p, img->stride_px);
    Plane gpl;
    {
        Stage st(ctx, "scanner");
        const double sb = s.scanner_lens_blur_px;
        const double su = s.unsharp_sigma_full * ctx.rho_tier;
        const double am = s.unsharp_amount;
        if (sb > 0.0) gaussian(ctx, rgb, rgb, Vec3{sb, sb, sb});
        if (su > 0.0 && am > 0.0) {
            gpl = make_plane(ctx.pool, w, h);
            gaussian(ctx, rgb, gpl, Vec3{su, su, su});
            e.unsharp = 1;
            e.lincomb_a = f32(1.0 + am);
            e.lincomb_b = f32(-am);
        }
    }
    {
        Stage st(ctx, "encode");
        dev::encode(rgb.data(), gpl ? gpl.data() : nullptr, img->dev, w, h, e, ctx.stream);
    }
    return false;
}


// ---- the adjoint of the render ------------------------------------------------------------------------

namespace {

// g := G^T g for the Gaussian of one sigma on every channel: the transposed FIR passes, or the
// block-parallel recursive kernels in transpose mode
void gaussian_adjoint(RenderCtx& ctx, Plane& g, double sigma) {
    const Branch br = blur_branch(sigma);
    if (br == Branch::Identity) return;
    if (br == Branch::Fir) {
        const bool no_iir[3] = {false, false, false};
        const FirTaps t = fir_taps(Vec3{sigma, sigma, sigma}, no_iir);
        if (t.r == 0) return;
        Plane tmp = make_plane(ctx.pool, g.w, g.h);
        dev::fir_pass_adjoint(g.data(), tmp.data(), g.w, g.h, t.r, t.taps[0], 0, ctx.stream);
        dev::fir_pass_adjoint(tmp.data(), g.data(), g.w, g.h, t.r, t.taps[0], 1, ctx.stream);
        return;
    }
    const std::vector<MixtureComponent> one{MixtureComponent{Vec3{1.0, 1.0, 1.0}, Vec3{sigma, sigma, sigma}}};
    if (!iir_mixture_mix(ctx, g, one, Vec3{0.0, 0.0, 0.0}, Vec3{1.0, 1.0, 1.0}, true))
        fail_unsupported("the transposed recursive blur needs the frame's lines in shared memory");
}

// d/dsigma of the blur of x by the Gaussian of one sigma on every channel, exact for the implemented
// filter: on the FIR branch the derivative of the normalised taps (fixed support) in either pass,
// dG x = H'(V x) + H(V' x); on the recursive branch the tangent of the Young-van Vliet recurrences
// along their coefficients' derivatives, row pass then column pass.
void gaussian_dsigma(RenderCtx& ctx, const Plane& x, double sigma, Plane& out_dot) {
    const uint32_t w = x.w, h = x.h;
    const Branch br = blur_branch(sigma);
    if (br == Branch::Identity) {
        cuda_check(cudaMemsetAsync(out_dot.data(), 0, out_dot.bytes(), ctx.stream), "memset");
        return;
    }
    if (br == Branch::Fir) {
        const bool no_iir[3] = {false, false, false};
        const FirTaps t = fir_taps(Vec3{sigma, sigma, sigma}, no_iir);
        FirTaps dt = t;
        const std::vector<double> d = gaussian_kernel_dsigma(sigma, 3.0);
        const int rd = int(d.size() / 2);
        for (int c = 0; c < 3; ++c)
            for (int i = -t.r; i <= t.r; ++i) dt.taps[c][t.r + i] = std::abs(i) <= rd ? f32(d[size_t(i + rd)]) : 0.0f;
        Plane a = make_plane(ctx.pool, w, h), b = make_plane(ctx.pool, w, h);
        const float one[3] = {1.0f, 1.0f, 1.0f};
        dev::fir_v(x.data(), a.data(), w, h, t, ctx.stream);
        dev::fir_h(a.data(), b.data(), b.data(), w, h, dt, ACC_NONE, one, ctx.stream);  // H'(V x)
        dev::fir_v(x.data(), a.data(), w, h, dt, ctx.stream);
        dev::fir_h(a.data(), out_dot.data(), b.data(), w, h, t, ACC_PLANE, one, ctx.stream);  // + H(V' x)
        return;
    }
    const bool all[3] = {true, true, true};
    const IirCoefs c = iir_coefs(Vec3{sigma, sigma, sigma}, all);
    IirCoefs dc = c;
    const IirCoefficients k = iir_coefficients_dsigma(sigma);
    for (int i = 0; i < 3; ++i) {
        dc.B[i] = k.B;
        dc.B1[i] = k.B1;
        dc.B2[i] = k.B2;
        dc.B3[i] = k.B3;
    }
    Plane work = make_plane(ctx.pool, w, h), work_dot = make_plane(ctx.pool, w, h);
    Plane rows = make_plane(ctx.pool, w, h), rows_dot = make_plane(ctx.pool, w, h), value = make_plane(ctx.pool, w, h);
    dev::iir_tangent(x.data(), nullptr, work.data(), work_dot.data(), rows.data(), rows_dot.data(), w, h, false, c, dc,
                     ctx.stream);
    dev::iir_tangent(rows.data(), rows_dot.data(), work.data(), work_dot.data(), value.data(), out_dot.data(), w, h, true,
                     c, dc, ctx.stream);
}

double common_sigma(const MixtureComponent& m) {
    if (!(m.sigma[0] == m.sigma[1] && m.sigma[1] == m.sigma[2]))
        fail_unsupported("the render's adjoint takes halation components with one sigma for the three channels");
    return m.sigma[0];
}

// g := a g + b sum_k w_k G_k^T g, the transpose of the mixture stage raw := a raw + b sum_k w_k G_k(raw)
void mixture_adjoint(RenderCtx& ctx, Plane& g, const std::vector<MixtureComponent>& comps, const Vec3& a,
                     const Vec3& b) {
    if (iir_mixture_mix(ctx, g, comps, a, b, true)) return;
    Plane acc = make_plane(ctx.pool, g.w, g.h);
    Plane t = make_plane(ctx.pool, g.w, g.h);
    for (size_t k = 0; k < comps.size(); ++k) {
        dev::copy(g.data(), t.data(), g.pixels(), ctx.stream);
        gaussian_adjoint(ctx, t, common_sigma(comps[k]));
        if (k == 0) lincomb(ctx, comps[k].weight, t, Vec3{0.0, 0.0, 0.0}, nullptr, acc);
        else lincomb(ctx, Vec3{1.0, 1.0, 1.0}, acc, comps[k].weight, &t, acc);
    }
    lincomb(ctx, a, g, b, &acc, g);
}

// The print stage in the adjoint's form, with the tangents of its per-print constants along
// print_exposure (k = print_exposure exactly) and the two filter shifts (binary64 central differences
// of the set-up, step 1e-4).
dev::VjpPrintArgs vjp_print_args(const Pipeline& p, const LiveParams& live, uint32_t n) {
    const PrintSetup& s = *p.print;
    const PrintRun r = compute_run(s, live);
    dev::VjpPrintArgs a{};
    std::memcpy(a.enl_eps, r.enl32.eps, sizeof a.enl_eps);
    std::memcpy(a.enl_beta, r.enl32.beta, sizeof a.enl_beta);
    std::memcpy(a.enl_wt, r.enl32.wt, sizeof a.enl_wt);
    std::memcpy(a.scan_eps, s.scan32.eps, sizeof a.scan_eps);
    std::memcpy(a.scan_beta, s.scan32.beta, sizeof a.scan_beta);
    std::memcpy(a.scan_wt, s.scan32.wt, sizeof a.scan_wt);
    for (int c = 0; c < 3; ++c) {
        a.g[c] = f32(r.g[c]);
        a.o[c] = f32(r.o[c]);
    }
    a.k_gain = r.k_gain;
    a.t_k[0] = 1.0f;
    constexpr double h = 1e-4;
    for (int j = 1; j < dev::kVjpPrintParams; ++j) {
        LiveParams lp = live, lm = live;
        double& vp = j == 1 ? lp.m_filter_shift : lp.y_filter_shift;
        double& vm = j == 1 ? lm.m_filter_shift : lm.y_filter_shift;
        vp += h;
        vm -= h;
        const PrintRun rp = compute_run(s, lp), rm = compute_run(s, lm);
        for (int i = 0; i < 3 * SPKB_NL; ++i) {
            a.t_eps[j][i] = f32((rp.eps_n[size_t(i)] - rm.eps_n[size_t(i)]) / (2.0 * h));
            a.t_wt[j][i] = f32((rp.w_n[size_t(i)] - rm.w_n[size_t(i)]) / (2.0 * h));
        }
        for (int l = 0; l < SPKB_NL; ++l) a.t_beta[j][l] = f32((rp.beta_n[size_t(l)] - rm.beta_n[size_t(l)]) / (2.0 * h));
        for (int c = 0; c < 3; ++c) {
            a.t_g[j][c] = f32((rp.g[c] - rm.g[c]) / (2.0 * h));
            a.t_o[j][c] = f32((rp.o[c] - rm.o[c]) / (2.0 * h));
        }
    }
    a.printed = s.scanned ? 0 : 1;
    a.paper = p.dev.paper.as<float>();
    a.paper_K = s.paper_K;
    if (!s.paper_tab.empty()) a.paper_grid = axis_grid(s.paper_tab.data(), s.paper_K, 1);
    std::memcpy(a.to_rgb, s.to_rgb, sizeof a.to_rgb);
    a.cam = s.cam_args;
    a.cmax = p.dev.cmax.as<float>();
    a.n = n;
    return a;
}

}  // namespace

void render_vjp(RenderCtx& ctx, const Pipeline& p, const LiveParams& live, const Plane& source, uint32_t film_seed,
                const std::optional<HalationOverride>& hov, float* y_out, const float* g_y, float* g_x,
                double* grad_params, uint32_t n_params) {
    const FilmSetup& f = *p.film;
    const PrintSetup& ps = *p.print;
    const uint32_t w = source.w, h = source.h;
    const size_t n = source.pixels();
    // ---- forward, keeping what the adjoint needs ----
    Plane H0 = make_plane(ctx.pool, w, h);
    const ExposeArgs ea = expose_args(f, n);
    dev::expose(source.data(), H0.data(), p.dev.table.as<float>(), p.dev.patches.as<float>(), ea, ctx.stream);
    const double s_lens = film_lens_blur_px(ctx, f);
    Plane H1 = H0;
    if (s_lens > 0.0) {
        H1 = make_plane(ctx.pool, w, h);
        gaussian(ctx, H0, H1, Vec3{s_lens, s_lens, s_lens});
    }
    const HalationPlan pl = film_halation(ctx, f, hov);
    Plane H2 = H1;  // after the scatter stage
    if (pl.scatter) {
        H2 = make_plane(ctx.pool, w, h);
        dev::copy(H1.data(), H2.data(), n, ctx.stream);
        HalationPlan only = pl;
        only.bounce = false;
        apply_halation(ctx, only, H2);
    }
    Plane H3 = H2;  // after the bounce stage: the exposure the develop stage reads
    if (pl.bounce) {
        H3 = make_plane(ctx.pool, w, h);
        dev::copy(H2.data(), H3.data(), n, ctx.stream);
        HalationPlan only = pl;
        only.scatter = false;
        apply_halation(ctx, only, H3);
    }
    DevBuffer counts = ctx.pool.acquire(n * 9 * sizeof(float));
    const DevelopPlan dp = develop_plan(ctx, p, w, film_seed, counts.as<float>());
    if (dp.grain && (dp.da.mode != 0 || dp.amount != 1.0))
        fail_unsupported("the render's adjoint takes sub-layer grain at full strength (or no grain)");
    if (f.couplers) fail_unsupported("the render's adjoint does not take DIR couplers");
    if (f.params.b(P::auto_exposure)) fail_unsupported("the render's adjoint does not take the auto-exposure meter");
    if (p.print->edr && !p.print->scanned) fail_unsupported("the render's adjoint does not take the EDR tone map");
    if (f.params.f(P::halation_boost_ev) != 0.0 || headroom_applies(f.halation))
        fail_unsupported("the render's adjoint does not take the highlight boost or headroom");
    if (!p.print->scanned && p.print->glare_draws()) fail_unsupported("the render's adjoint does not take print glare");
    if (f.decode || !geometry_identity(f.params))
        fail_unsupported("the render's adjoint does not take the input transfer decode or a geometry");
    Plane G = make_plane(ctx.pool, w, h);
    dev::develop(H3.data(), G.data(), dp.da, w, h, ctx.stream);
    Plane neg = G;
    if (dp.grain && dp.final_blur > 0.0) {
        neg = make_plane(ctx.pool, w, h);
        gaussian(ctx, G, neg, Vec3{dp.final_blur, dp.final_blur, dp.final_blur});
    }
    const dev::VjpPrintArgs va = vjp_print_args(p, live, uint32_t(n));
    PrintArgs pa{};
    {
        const PrintRun r = compute_run(ps, live);
        pa.enl = spectral_pairs(r.enl32);
        pa.scan = spectral_pairs(ps.scan32);
        for (int c = 0; c < 3; ++c) {
            pa.g[c] = f32(r.g[c]);
            pa.o[c] = f32(r.o[c]);
        }
        pa.k_gain = r.k_gain;
        pa.printed = va.printed;
        pa.paper = va.paper;
        pa.paper_K = va.paper_K;
        pa.paper_grid = va.paper_grid;
        std::memcpy(pa.to_rgb, ps.to_rgb, sizeof pa.to_rgb);
        pa.cam = ps.cam_args;
        pa.cmax = va.cmax;
        pa.n = uint32_t(n);
    }
    Plane P = make_plane(ctx.pool, w, h);
    dev::print(neg.data(), P.data(), pa, ctx.stream);
    const double sb = ps.scanner_lens_blur_px, su = ps.unsharp_sigma_full * ctx.rho_tier, am = ps.unsharp_amount;
    const bool unsharp = su > 0.0 && am > 0.0;
    Plane B = P;
    if (sb > 0.0) {
        B = make_plane(ctx.pool, w, h);
        gaussian(ctx, P, B, Vec3{sb, sb, sb});
    }
    Plane Y = B;
    if (unsharp) {
        Plane Gs = make_plane(ctx.pool, w, h);
        gaussian(ctx, B, Gs, Vec3{su, su, su});
        Y = make_plane(ctx.pool, w, h);
        lincomb(ctx, Vec3{1.0 + am, 1.0 + am, 1.0 + am}, B, Vec3{-am, -am, -am}, &Gs, Y);
    }
    if (y_out) cuda_check(cudaMemcpyAsync(y_out, Y.data(), Y.bytes(), cudaMemcpyDeviceToDevice, ctx.stream), "copy");
    if (!g_y) return;

    // ---- adjoint ----
    const uint32_t ncomp = hov ? uint32_t(hov->comps.size()) : 0u;
    constexpr uint32_t kNodes = 3 * dev::kVjpCurveNodes;
    const uint32_t n_all = dev::kVjpPrintParams + 2 * ncomp + kNodes;
    // device accumulators: print parameters | per component [weight 3 | sigma 3] | curve parameters
    constexpr size_t kAcc = dev::kVjpPrintParams + 6 * SPKB_MAX_COMPONENTS + kNodes;
    DevBuffer dparams = ctx.pool.acquire(sizeof(double) * kAcc);
    cuda_check(cudaMemsetAsync(dparams.ptr(), 0, sizeof(double) * kAcc, ctx.stream), "memset");
    double* d_print = dparams.as<double>();
    double* d_dots = d_print + dev::kVjpPrintParams;  // [k][weight 3 | sigma 3]
    double* d_nodes = d_dots + 6 * SPKB_MAX_COMPONENTS;
    Plane g = make_plane(ctx.pool, w, h);
    cuda_check(cudaMemcpyAsync(g.data(), g_y, g.bytes(), cudaMemcpyDeviceToDevice, ctx.stream), "copy");
    if (unsharp) {  // g_B = (1 + a) g_Y - a Gs^T g_Y
        Plane t = make_plane(ctx.pool, w, h);
        dev::copy(g.data(), t.data(), n, ctx.stream);
        gaussian_adjoint(ctx, t, su);
        lincomb(ctx, Vec3{1.0 + am, 1.0 + am, 1.0 + am}, g, Vec3{-am, -am, -am}, &t, g);
    }
    if (sb > 0.0) gaussian_adjoint(ctx, g, sb);  // g_P
    Plane gn = make_plane(ctx.pool, w, h);
    dev::vjp_print(neg.data(), g.data(), gn.data(), d_print, va, ctx.stream);
    if (dp.grain && dp.final_blur > 0.0) gaussian_adjoint(ctx, gn, dp.final_blur);  // g_G
    dev::vjp_develop(H3.data(), counts.as<float>(), gn.data(), g.data(), d_nodes, dp.da, w, h, ctx.stream);  // g_H3
    if (pl.bounce) {
        if (hov) {  // the override's weights and sigmas, from the exposure entering the bounce stage (H2)
            Plane Gk = make_plane(ctx.pool, w, h);
            for (uint32_t k = 0; k < ncomp; ++k) {
                const double sg = common_sigma(hov->comps[k]);
                gaussian(ctx, H2, Gk, Vec3{sg, sg, sg});
                dev::dot3(g.data(), Gk.data(), n, d_dots + 6 * k, ctx.stream);
                gaussian_dsigma(ctx, H2, sg, Gk);
                dev::dot3(g.data(), Gk.data(), n, d_dots + 6 * k + 3, ctx.stream);
            }
        }
        mixture_adjoint(ctx, g, pl.bounce_comps, pl.mix_a, pl.mix_b);  // g_H2
    }
    if (pl.scatter) mixture_adjoint(ctx, g, pl.scatter_comps, pl.scatter_a, pl.scatter_b);  // g_H1
    if (s_lens > 0.0) gaussian_adjoint(ctx, g, s_lens);  // g_H0
    dev::vjp_expose(source.data(), g.data(), g_x, p.dev.table.as<float>(), ea, ctx.stream);
    double hp[kAcc];
    cuda_check(cudaMemcpyAsync(hp, dparams.ptr(), sizeof hp, cudaMemcpyDeviceToHost, ctx.stream), "copy");
    cuda_check(cudaStreamSynchronize(ctx.stream), "render adjoint");
    if (!grad_params) return;
    std::vector<double> all(n_all, 0.0);
    for (int j = 0; j < dev::kVjpPrintParams; ++j) all[size_t(j)] = hp[j];
    for (uint32_t k = 0; k < ncomp; ++k) {
        const double* dk = hp + dev::kVjpPrintParams + 6 * k;
        double gw = 0.0, gs = 0.0;
        for (int c = 0; c < 3; ++c) {
            gw += pl.mix_b[c] * dk[c];
            gs += pl.mix_b[c] * hov->comps[k].weight[c] * dk[3 + c];
        }
        all[dev::kVjpPrintParams + k] = gw;
        all[dev::kVjpPrintParams + ncomp + k] = gs;
    }
    for (uint32_t i = 0; i < kNodes; ++i)
        all[dev::kVjpPrintParams + 2 * ncomp + i] = hp[dev::kVjpPrintParams + 6 * SPKB_MAX_COMPONENTS + i];
    for (uint32_t j = 0; j < n_params; ++j) grad_params[j] = j < n_all ? all[j] : 0.0;
}

}  // namespace spkb
