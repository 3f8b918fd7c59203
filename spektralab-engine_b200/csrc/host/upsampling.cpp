// The spectral upsampling table of the film set-up (reference src/film/setup.cpp:133-257): for every node
// of the L x L chromaticity grid, the three film layers' responses to the node's reflectance spectrum, with
// the input gamut compression baked in.
//
// Steps, each a function below:
//   1. layer weights: the layer sensitivities, optionally shaped by the stock's UV / IR adaptation window
//      and renormalised so the window keeps each layer's response to the reference illuminant;
//   2. node responses: the weights contracted with each node's 81-bin spectrum;
//   3. gamut compression: each grid node's chromaticity is pulled toward the illuminant's white along the
//      ray from the white, its distance measured in units of the distance to the spectrum locus (the
//      polygon of the CIE 1931 chromaticities from 380 to 700 nm, closed by the purple line) and passed
//      through a soft knee, so out-of-locus chromaticities land inside it;
//   4. resampling: the node responses read back bilinearly at the compressed chromaticity's grid
//      coordinates.
// The floating-point expressions keep the reference's operation order (the narrowed table is pinned bit
// for bit against it); the decomposition, names and messages are this file's.
#include <algorithm>
#include <cmath>
#include <limits>

#include "setup.hpp"
#include "status.hpp"

namespace spkb {

namespace {

constexpr size_t kBins = 81;        // 380..780 nm at 5 nm
constexpr size_t kLocusBins = 65;   // 380..700 nm: the locus polygon's vertices before the purple line

struct Point {
    double x, y;
};

// grid chromaticity coordinates (t0, t1) of the xy point: t0 = (1 - x)^2, t1 = y / (1 - x), both clipped
// to [0, 1]; the inverse of the grid's parametrisation x = 1 - sqrt(t0), y = t1 sqrt(t0)
std::array<double, 2> grid_coords(Point p) {
    auto unit = [](double v) { return std::min(std::max(v, 0.0), 1.0); };
    const double o = 1.0 - p.x;
    return {unit(o * o), unit(p.y / std::max(o, 1e-10))};
}

// 1. the layer weights, bin-major (3 per bin)
std::array<double, 243> layer_weights(const std::array<double, 243>& sens, const std::vector<double>& window,
                                      const Spectrum& light) {
    std::array<double, 243> w = sens;
    if (window.empty()) return w;
    if (window.size() != 4)
        fail_user("film stock: its spectral adaptation window has " + std::to_string(window.size()) +
                  " parameters; only the (uv centre, uv width, ir centre, ir width) form is supported");
    const double uv_at = window[0], uv_width = window[1], ir_at = window[2], ir_width = window[3];
    const double root2 = std::sqrt(2.0);
    std::array<double, kBins> pass{};
    for (size_t b = 0; b < kBins; ++b) {
        const double nm = 380.0 + 5.0 * double(b);
        const double rise = 0.5 * (1.0 + std::erf((nm - uv_at) / (uv_width * root2)));
        const double fall = 0.5 * (1.0 - std::erf((nm - ir_at) / (ir_width * root2)));
        pass[b] = rise * fall;
    }
    for (size_t c = 0; c < 3; ++c) {
        double shaped = 0.0, plain = 0.0;
        for (size_t b = 0; b < kBins; ++b) {
            shaped += sens[3 * b + c] * pass[b] * light[b];
            plain += sens[3 * b + c] * light[b];
        }
        const double keep = shaped / plain;
        for (size_t b = 0; b < kBins; ++b) w[3 * b + c] = sens[3 * b + c] * pass[b] / keep;
    }
    return w;
}

// 2. every node's response, node-major (3 per node)
std::vector<double> node_responses(const std::vector<double>& spectra, const std::array<double, 243>& w, size_t nodes) {
    std::vector<double> out(nodes * 3);
    for (size_t n = 0; n < nodes; ++n) {
        const double* r = spectra.data() + n * kBins;
        double acc[3] = {0.0, 0.0, 0.0};
        for (size_t b = 0; b < kBins; ++b)
            for (size_t c = 0; c < 3; ++c) acc[c] += r[b] * w[3 * b + c];
        for (size_t c = 0; c < 3; ++c) out[3 * n + c] = acc[c];
    }
    return out;
}

// 3. the spectrum locus as a closed polygon, and the distance from an inner point to it along a ray
class Locus {
public:
    explicit Locus(const std::vector<double>& cmf) {
        for (size_t b = 0; b < kLocusBins; ++b) {
            const double X = cmf[3 * b], Y = cmf[3 * b + 1], Z = cmf[3 * b + 2];
            const double sum = std::max(X + Y + Z, 1e-12);
            v_.push_back({X / sum, Y / sum});
        }
        v_.push_back(v_.front());  // the purple line
    }

    // the smallest positive s with from + s dir on an edge (dir a unit vector); +inf when no edge is hit
    double exit_distance(Point from, Point dir) const {
        double best = std::numeric_limits<double>::infinity();
        for (size_t k = 0; k + 1 < v_.size(); ++k) {
            const Point a = v_[k], b = v_[k + 1];
            const double ex = b.x - a.x, ey = b.y - a.y;
            const double cross = dir.x * ey - dir.y * ex;
            if (std::fabs(cross) <= 1e-12) continue;  // parallel to the edge
            const double ox = from.x - a.x, oy = from.y - a.y;
            const double along_ray = (-ox * ey + oy * ex) / cross;
            const double along_edge = (-ox * dir.y + oy * dir.x) / cross;
            if (along_edge >= 0.0 && along_edge <= 1.0 && along_ray > 1e-9 && along_ray < best) best = along_ray;
        }
        return best;
    }

private:
    std::vector<Point> v_;
};

// the radius knee: r / (1 + r^6)^(1/6), the identity near 0 and approaching 1 for large r
double soft_clip(double r) { return r / std::pow(1.0 + std::pow(r, 6.0), 1.0 / 6.0); }

// the grid point's chromaticity pulled inside the locus (unchanged at the white itself)
Point compress(Point p, Point white, const Locus& locus) {
    const double dx = p.x - white.x, dy = p.y - white.y;
    const double dist = std::sqrt(dx * dx + dy * dy);
    if (dist < 1e-9) return p;
    const double norm = std::max(dist, 1e-12);
    const Point dir{dx / norm, dy / norm};
    const double edge = locus.exit_distance(white, dir);
    const double r = dist / std::max(edge, 1e-12);
    const double scaled = r > 0.0 ? soft_clip(r) : r;
    return {white.x + dir.x * scaled * edge, white.y + dir.y * scaled * edge};
}

// 4. bilinear read of the node responses at grid coordinates (t0, t1)
struct GridCell {
    uint32_t lo, hi;
    double frac;
};
GridCell grid_cell(double t, uint32_t L) {
    const double last = double(L - 1);
    double u = t * last;
    if (!(u > 0.0)) u = 0.0;
    if (u > last) u = last;
    const double whole = std::floor(u);
    const uint32_t lo = uint32_t(whole);
    return {lo, std::min(lo + 1, L - 1), u - whole};
}

}  // namespace

std::vector<double> spectral_upsampling_table(const Blob& blob, const std::array<double, 243>& sens,
                                              const std::vector<double>& window, const Spectrum& light,
                                              uint32_t* L_out) {
    const BlobEntry* grid = blob.find("hanatos/spectra_lut");
    if (!grid || grid->ndim != 3 || grid->dims[0] != grid->dims[1] || grid->dims[2] != kBins || grid->dims[0] < 2)
        fail_user("spectral upsampling: the resources need a square grid of 81-bin reflectance spectra "
                  "(hanatos/spectra_lut, L x L x 81, L >= 2)");
    const uint32_t L = grid->dims[0];
    *L_out = L;
    const size_t nodes = size_t(L) * L;
    const std::vector<double> responses = node_responses(blob.f64("hanatos/spectra_lut"),
                                                         layer_weights(sens, window, light), nodes);
    const std::vector<double> cmf = blob.f64("colour/cmfs_1931_2deg");
    if (cmf.size() != 3 * kBins) fail_user("spectral upsampling: colour/cmfs_1931_2deg needs 81 rows of X, Y, Z");
    Point white{};
    {
        double X = 0.0, Y = 0.0, Z = 0.0;
        for (size_t b = 0; b < kBins; ++b) {
            X += light[b] * cmf[3 * b];
            Y += light[b] * cmf[3 * b + 1];
            Z += light[b] * cmf[3 * b + 2];
        }
        const double sum = X + Y + Z;
        white = {X / sum, Y / sum};
    }
    const Locus locus(cmf);
    const double last = double(L - 1);
    std::vector<double> table(nodes * 3);
    for (uint32_t i = 0; i < L; ++i)
        for (uint32_t j = 0; j < L; ++j) {
            const double root = std::sqrt(double(i) / last);
            const Point node{1.0 - root, (double(j) / last) * root};
            const std::array<double, 2> t = grid_coords(compress(node, white, locus));
            const GridCell a = grid_cell(t[0], L), b = grid_cell(t[1], L);
            const double* r00 = &responses[3 * (size_t(a.lo) * L + b.lo)];
            const double* r01 = &responses[3 * (size_t(a.lo) * L + b.hi)];
            const double* r10 = &responses[3 * (size_t(a.hi) * L + b.lo)];
            const double* r11 = &responses[3 * (size_t(a.hi) * L + b.hi)];
            double* out = &table[3 * (size_t(i) * L + j)];
            const double ua = 1.0 - a.frac, ub = 1.0 - b.frac;
            for (size_t c = 0; c < 3; ++c)
                out[c] = r00[c] * ua * ub + r01[c] * ua * b.frac + r10[c] * a.frac * ub + r11[c] * a.frac * b.frac;
        }
    return table;
}

}  // namespace spkb
