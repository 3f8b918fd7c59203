#include "resources.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

#include "status.hpp"

namespace spkb {

namespace {
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();
constexpr size_t kHeader = 16, kEntry = 104;

uint32_t rd32(const uint8_t* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
uint64_t rd64(const uint8_t* p) {
    uint64_t v;
    std::memcpy(&v, p, 8);
    return v;
}
size_t dtype_size(uint32_t t) {
    static const size_t s[5] = {8, 4, 2, 4, 1};
    return s[t];
}
double half_to_double(uint16_t h) {
    const int sign = (h >> 15) & 1, e = (h >> 10) & 0x1F, m = h & 0x3FF;
    double v;
    if (e == 0) v = std::ldexp(double(m), -24);
    else if (e == 31) v = m ? kNaN : std::numeric_limits<double>::infinity();
    else v = std::ldexp(double(m | 0x400), e - 25);
    return sign ? -v : v;
}
}  // namespace

uint64_t BlobEntry::count() const {
    uint64_t n = 1;
    for (uint32_t i = 0; i < ndim; ++i) n *= dims[i];
    return n;
}

Blob::~Blob() {
    if (data_) munmap(const_cast<uint8_t*>(data_), size_);
}

std::shared_ptr<const Blob> Blob::open(const std::filesystem::path& file) {
    const int fd = ::open(file.c_str(), O_RDONLY | O_CLOEXEC);
    if (fd < 0) fail_io("cannot open '" + file.string() + "'");
    struct stat st {};
    if (fstat(fd, &st) != 0) {
        ::close(fd);
        fail_io("cannot stat '" + file.string() + "'");
    }
    const size_t size = size_t(st.st_size);
    if (size < kHeader) {
        ::close(fd);
        fail_io("constants blob: truncated header");
    }
    void* m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    ::close(fd);
    if (m == MAP_FAILED) fail_io("cannot map '" + file.string() + "'");
    std::shared_ptr<Blob> b(new Blob());
    b->data_ = static_cast<const uint8_t*>(m);
    b->size_ = size;
    const uint8_t* d = b->data_;
    if (std::memcmp(d, "SPKR", 4) != 0) fail_io("constants blob: wrong magic");
    if (rd32(d + 4) != 1) fail_io("constants blob: unsupported version " + std::to_string(rd32(d + 4)));
    const uint32_t count = rd32(d + 8);
    if (kHeader + uint64_t(count) * kEntry > size) fail_io("constants blob: truncated entry table");
    bool any_cat = false;
    for (uint32_t i = 0; i < count; ++i) {
        const uint8_t* e = d + kHeader + size_t(i) * kEntry;
        BlobEntry en;
        size_t len = 0;
        while (len < 64 && e[len] != 0) ++len;
        if (len == 64) fail_io("constants blob: entry " + std::to_string(i) + " name is not NUL-terminated");
        en.name.assign(reinterpret_cast<const char*>(e), len);
        en.dtype = rd32(e + 64);
        if (en.dtype > 4) fail_io("constants blob: entry '" + en.name + "' has an unknown dtype");
        en.ndim = rd32(e + 68);
        if (en.ndim < 1 || en.ndim > 4) fail_io("constants blob: entry '" + en.name + "' ndim out of 1..4");
        for (int k = 0; k < 4; ++k) en.dims[k] = rd32(e + 72 + 4 * k);
        for (uint32_t k = en.ndim; k < 4; ++k)
            if (en.dims[k] != 0) fail_io("constants blob: entry '" + en.name + "' has a non-zero unused dimension");
        en.offset = rd64(e + 88);
        en.nbytes = rd64(e + 96);
        if (en.offset % 8 != 0) fail_io("constants blob: entry '" + en.name + "' offset is not 8-aligned");
        if (en.offset > size || en.nbytes > size - en.offset)
            fail_io("constants blob: entry '" + en.name + "' runs past the end of the file");
        en.size_ok = en.count() * dtype_size(en.dtype) == en.nbytes;
        if (en.name.rfind("colour/cat/", 0) == 0) any_cat = true;
        b->entries_[en.name] = std::move(en);
    }
    for (const char* r : {"spectral/wavelengths", "colour/cmfs_1931_2deg", "colour/cmfs_lms", "colour/matrix_16",
                          "colour/mallett_srgb_basis", "hanatos/spectra_lut"}) {
        const BlobEntry* en = b->find(r);
        if (!en) fail_io(std::string("constants blob: required entry '") + r + "' is missing");
        if (!en->size_ok) fail_io(std::string("constants blob: required entry '") + r + "' does not match its shape");
    }
    const BlobEntry* wl = b->find("spectral/wavelengths");
    if (wl->ndim != 1 || wl->dims[0] != 81) fail_io("constants blob: 'spectral/wavelengths' must have 81 samples");
    if (!any_cat) fail_io("constants blob: no 'colour/cat/*' entry");
    return b;
}

const BlobEntry* Blob::find(std::string_view name) const {
    auto it = entries_.find(name);
    return it == entries_.end() ? nullptr : &it->second;
}

std::vector<double> Blob::f64(std::string_view name) const {
    const BlobEntry* e = find(name);
    if (!e) fail_user("constants blob has no entry '" + std::string(name) + "'");
    if (!e->size_ok) fail_user("constants blob entry '" + std::string(name) + "' does not match its shape");
    const uint8_t* p = data_ + e->offset;
    const size_t n = size_t(e->count());
    std::vector<double> out(n);
    for (size_t i = 0; i < n; ++i) {
        switch (e->dtype) {
            case 0: {
                double v;
                std::memcpy(&v, p + 8 * i, 8);
                out[i] = v;
                break;
            }
            case 1: {
                float v;
                std::memcpy(&v, p + 4 * i, 4);
                out[i] = v;
                break;
            }
            case 2: {
                uint16_t v;
                std::memcpy(&v, p + 2 * i, 2);
                out[i] = half_to_double(v);
                break;
            }
            case 3: {
                int32_t v;
                std::memcpy(&v, p + 4 * i, 4);
                out[i] = v;
                break;
            }
            default: out[i] = p[i];
        }
    }
    return out;
}

// ---- colour ---------------------------------------------------------------------------------------

namespace {
constexpr std::string_view kSpaceNames[] = {"sRGB",         "Display P3",    "ProPhoto RGB", "Adobe RGB (1998)",
                                            "ITU-R BT.709", "ITU-R BT.2020", "ACEScg",       "ACES2065-1"};
constexpr Cctf kSpaceModes[] = {Cctf::SRGB, Cctf::SRGB, Cctf::ProPhoto, Cctf::Adobe,
                                Cctf::BT709, Cctf::BT709, Cctf::Identity, Cctf::Identity};

template <size_t N>
bool blob_array(const Blob& b, const std::string& name, std::array<double, N>& out) {
    const BlobEntry* e = b.find(name);
    if (!e || !e->size_ok || e->count() != N) return false;
    const std::vector<double> v = b.f64(name);
    for (size_t i = 0; i < N; ++i) out[i] = v[i];
    return true;
}

std::optional<Spectrum> blob_spectrum(const Blob& b, const std::string& name) {
    const BlobEntry* e = b.find(name);
    if (!e || !e->size_ok || e->ndim != 1 || e->dims[0] != 81) return std::nullopt;
    Spectrum s{};
    const std::vector<double> v = b.f64(name);
    for (size_t i = 0; i < 81; ++i) s[i] = v[i];
    return s;
}

std::optional<Spectrum> raw_illuminant(const Blob& b, std::string_view name) {
    if (name.size() > 2 && name.substr(0, 2) == "BB") {
        const std::string num(name.substr(2));
        char* end = nullptr;
        const double t = std::strtod(num.c_str(), &end);
        if (end == num.c_str() || !std::isfinite(t) || !(t > 0)) return std::nullopt;
        return blackbody(t);
    }
    if (name == "T") return blob_spectrum(b, "colour/sd_light_source/Incandescent");
    if (name == "K75P") return blob_spectrum(b, "colour/sd_light_source/Kinoton 75P");
    if (name == "TH-KG3" || name == "TH-KG3-L") {
        auto kg3 = blob_spectrum(b, "filters/kg3");
        if (!kg3) return std::nullopt;
        Spectrum s = blackbody(3400.0);
        for (size_t i = 0; i < 81; ++i) s[i] *= (*kg3)[i];
        if (name == "TH-KG3-L") {
            auto lens = blob_spectrum(b, "filters/lens_canon");
            if (!lens) return std::nullopt;
            for (size_t i = 0; i < 81; ++i) s[i] *= (*lens)[i];
        }
        return s;
    }
    if (auto s = blob_spectrum(b, "colour/sd_illuminant/" + std::string(name))) return s;
    return blob_spectrum(b, "colour/sd_light_source/" + std::string(name));
}

bool allclose(const std::array<double, 2>& a, const std::array<double, 2>& b) {
    for (size_t k = 0; k < 2; ++k)
        if (!(std::fabs(a[k] - b[k]) <= 1e-8 + 1e-5 * std::fabs(b[k]))) return false;
    return true;
}
}  // namespace

std::optional<Cctf> cctf_of(std::string_view name) {
    for (size_t i = 0; i < 8; ++i)
        if (kSpaceNames[i] == name) return kSpaceModes[i];
    return std::nullopt;
}

std::optional<ColourSpace> colour_space(const Blob& b, std::string_view name) {
    auto mode = cctf_of(name);
    if (!mode) return std::nullopt;
    ColourSpace cs;
    cs.name = std::string(name);
    cs.cctf = *mode;
    const std::string p = "colour/cs/" + cs.name + "/";
    if (!blob_array(b, p + "primaries", cs.primaries) || !blob_array(b, p + "whitepoint", cs.whitepoint) ||
        !blob_array(b, p + "matrix_RGB_to_XYZ", cs.rgb_to_xyz) || !blob_array(b, p + "matrix_XYZ_to_RGB", cs.xyz_to_rgb))
        return std::nullopt;
    return cs;
}

std::optional<Mat3> cat_matrix(const Blob& b, std::string_view name) {
    Mat3 m{};
    if (!blob_array(b, "colour/cat/" + std::string(name), m)) return std::nullopt;
    return m;
}

// Planck's law with the radiation constants of the reference (c1 = 3.741771e-16, c2 = 1.4388e-2,
// wavelength in metres): s = (c1 / (pi l^5)) / expm1(c2 / (l T)), unnormalised.
Spectrum blackbody(double kelvin) {
    constexpr double c1 = 3.741771e-16, c2 = 1.4388e-2, n = 1.0;
    Spectrum s{};
    for (size_t i = 0; i < 81; ++i) {
        const double lam = (380.0 + 5.0 * double(i)) * 1e-9;
        s[i] = (c1 / (M_PI * n * n * std::pow(lam, 5))) / std::expm1(c2 / (n * lam * kelvin));
    }
    return s;
}

std::optional<Spectrum> illuminant(const Blob& b, std::string_view name) {
    auto s = raw_illuminant(b, name);
    if (!s) return std::nullopt;
    double sum = 0.0;
    for (double x : *s) sum += x;
    const double mean = sum / 81.0;
    for (double& x : *s) x /= mean;
    return s;
}

std::array<double, 2> chromaticity(const Blob& b, const Spectrum& s) {
    const std::vector<double> cmf = b.f64("colour/cmfs_1931_2deg");
    double X = 0, Y = 0, Z = 0;
    for (size_t i = 0; i < 81; ++i) {
        X += s[i] * cmf[3 * i];
        Y += s[i] * cmf[3 * i + 1];
        Z += s[i] * cmf[3 * i + 2];
    }
    const double t = X + Y + Z;
    return {X / t, Y / t};
}

Mat3 mat3_mul(const Mat3& a, const Mat3& b) {
    Mat3 r{};
    for (size_t i = 0; i < 3; ++i)
        for (size_t j = 0; j < 3; ++j) {
            double s = 0.0;
            for (size_t k = 0; k < 3; ++k) s += a[3 * i + k] * b[3 * k + j];
            r[3 * i + j] = s;
        }
    return r;
}

Vec3 mat3_apply(const Mat3& m, const Vec3& v) {
    Vec3 r{};
    for (size_t i = 0; i < 3; ++i) {
        double s = 0.0;
        for (size_t k = 0; k < 3; ++k) s += m[3 * i + k] * v[k];
        r[i] = s;
    }
    return r;
}

Mat3 mat3_inverse(const Mat3& m) {
    const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    const double A0 = e * i - f * h, B0 = -(d * i - f * g), C0 = d * h - e * g;
    const double r = 1.0 / (a * A0 + b * B0 + c * C0);
    return {A0 * r, -(b * i - c * h) * r, (b * f - c * e) * r, B0 * r, (a * i - c * g) * r,
            -(a * f - c * d) * r, C0 * r, -(a * h - b * g) * r, (a * e - b * d) * r};
}

Vec3 xy_to_XYZ(const std::array<double, 2>& xy) { return {xy[0] / xy[1], 1.0, (1.0 - xy[0] - xy[1]) / xy[1]}; }

std::optional<Mat3> von_kries(const std::array<double, 2>& src, const std::array<double, 2>& dst, const Mat3& cone,
                              Guard g) {
    const bool close = g == Guard::Source ? allclose(dst, src) : allclose(src, dst);
    if (close) return std::nullopt;
    const Vec3 rs = mat3_apply(cone, xy_to_XYZ(src));
    const Vec3 rt = mat3_apply(cone, xy_to_XYZ(dst));
    Mat3 dg{};
    for (size_t k = 0; k < 3; ++k) dg[4 * k] = rt[k] / rs[k];
    return mat3_mul(mat3_mul(mat3_inverse(cone), dg), cone);
}

// ---- numeric --------------------------------------------------------------------------------------

double nanmin_strided(const double* p, size_t n, size_t stride) {
    double m = kNaN;
    for (size_t i = 0; i < n; ++i) {
        const double x = p[i * stride];
        if (std::isnan(x)) continue;
        if (std::isnan(m) || x < m) m = x;
    }
    return m;
}

double nanmax_strided(const double* p, size_t n, size_t stride) {
    double m = kNaN;
    for (size_t i = 0; i < n; ++i) {
        const double x = p[i * stride];
        if (std::isnan(x)) continue;
        if (std::isnan(m) || x > m) m = x;
    }
    return m;
}

double nanmean(const double* p, size_t n) {
    double s = 0.0;
    size_t k = 0;
    for (size_t i = 0; i < n; ++i) {
        if (std::isnan(p[i])) continue;
        s += p[i];
        ++k;
    }
    return k ? s / double(k) : kNaN;
}

double interp(double v, const std::vector<double>& x, const std::vector<double>& y) {
    const size_t k = x.size();
    if (std::isnan(v)) return kNaN;
    if (v <= x[0]) return y[0];
    if (v >= x[k - 1]) return y[k - 1];
    size_t lo = 0, hi = k;
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (x[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    size_t j = lo == 0 ? 0 : lo - 1;
    if (j + 1 >= k) j = k - 2;
    const double dx = x[j + 1] - x[j];
    if (dx == 0.0) return y[j];
    return y[j] + (v - x[j]) / dx * (y[j + 1] - y[j]);
}

// ---- profiles ---------------------------------------------------------------------------------------

namespace {

struct Ctx {
    std::string id;
    [[noreturn]] void bad(const std::string& what) const { fail_user("profile '" + id + "': " + what); }
};

json::Value parse_file(const std::filesystem::path& p, const Ctx& c) {
    std::ifstream f(p, std::ios::binary);
    if (!f) c.bad("cannot read '" + p.string() + "'");
    std::ostringstream ss;
    ss << f.rdbuf();
    try {
        return json::parse(ss.str());
    } catch (const json::ParseError& e) {
        c.bad(e.what());
    }
}

double num_or_nan(const json::Value& v, const Ctx& c, const char* key) {
    if (v.is_number()) return v.as_number();
    if (v.is_null()) return kNaN;
    c.bad(std::string("'") + key + "' holds a non-numeric element");
}

std::vector<double> vec(const json::Value& v, size_t n, const Ctx& c, const char* key) {
    if (!v.is_array()) c.bad(std::string("'") + key + "' must be an array");
    const auto& a = v.as_array();
    if (n && a.size() != n) c.bad(std::string("'") + key + "' must have " + std::to_string(n) + " values");
    std::vector<double> out;
    out.reserve(a.size());
    for (const auto& e : a) out.push_back(num_or_nan(e, c, key));
    return out;
}

Mat mat(const json::Value& v, size_t rows, size_t cols, const Ctx& c, const char* key) {
    if (!v.is_array()) c.bad(std::string("'") + key + "' must be an array");
    const auto& a = v.as_array();
    if (rows && a.size() != rows) c.bad(std::string("'") + key + "' must have " + std::to_string(rows) + " rows");
    if (a.empty()) c.bad(std::string("'") + key + "' is empty");
    Mat m;
    m.rows = a.size();
    m.cols = cols;
    for (const auto& r : a) {
        if (!r.is_array() || r.as_array().size() != cols)
            c.bad(std::string("'") + key + "' must have rows of " + std::to_string(cols) + " values");
        for (const auto& e : r.as_array()) m.v.push_back(num_or_nan(e, c, key));
    }
    return m;
}

Mat mat_any(const json::Value& v, const Ctx& c, const char* key) {
    if (!v.is_array() || v.as_array().empty() || !v.as_array()[0].is_array())
        c.bad(std::string("'") + key + "' must be a non-empty array of arrays");
    return mat(v, 0, v.as_array()[0].as_array().size(), c, key);
}

void read_info(const json::Value& info, Profile& p) {
    auto str = [&](const char* k, std::string& dst) {
        if (const json::Value* v = info.find(k); v && v->is_string()) dst = v->as_string();
    };
    str("type", p.type);
    str("support", p.support);
    str("use", p.use);
    str("antihalation", p.antihalation);
    str("reference_illuminant", p.reference_illuminant);
    str("viewing_illuminant", p.viewing_illuminant);
}

void read_data(const json::Value& data, Profile& p, const Ctx& c) {
    if (!data.is_object()) c.bad("'data' must be an object");
    auto req = [&](const char* k) -> const json::Value& {
        const json::Value* v = data.find(k);
        if (!v) c.bad(std::string("data.") + k + " is missing");
        return *v;
    };
    const std::vector<double> wl = vec(req("wavelengths"), 81, c, "wavelengths");
    for (size_t i = 0; i < 81; ++i)
        if (wl[i] != 380.0 + 5.0 * double(i)) c.bad("wavelengths must be 380, 385, ..., 780");
    p.log_sensitivity = mat(req("log_sensitivity"), 81, 3, c, "log_sensitivity");
    p.channel_density = mat(req("channel_density"), 81, 3, c, "channel_density");
    p.base_density = vec(req("base_density"), 81, c, "base_density");
    p.log_exposure = vec(req("log_exposure"), 0, c, "log_exposure");
    const size_t K = p.log_exposure.size();
    if (K < 2) c.bad("log_exposure needs at least 2 points");
    p.density_curves = mat(req("density_curves"), K, 3, c, "density_curves");
    if (const json::Value* v = data.find("density_curves_layers")) {
        if (!v->is_array() || v->as_array().size() != K) c.bad("density_curves_layers must be K x 3 x 3");
        for (const auto& row : v->as_array()) {
            const Mat m = mat(row, 3, 3, c, "density_curves_layers");
            p.layers.insert(p.layers.end(), m.v.begin(), m.v.end());
        }
    }
    if (const json::Value* v = data.find("edr_tone_map")) {
        // validated as the reference does (src/res/profile.cpp:113-141)
        if (!v->is_object()) c.bad("'edr_tone_map' must be an object");
        const json::Value* ver = v->find("version");
        if (!ver || !ver->is_number() || ver->as_number() != 1.0) c.bad("edr_tone_map.version must be 1");
        const json::Value* dom = v->find("domain_log2_y");
        if (!dom) c.bad("edr_tone_map.domain_log2_y is missing");
        const std::vector<double> d = vec(*dom, 2, c, "edr_tone_map.domain_log2_y");
        Profile::Edr e;
        e.lo = d[0];
        e.hi = d[1];
        if (!(e.hi > e.lo)) c.bad("edr_tone_map.domain_log2_y needs hi > lo");
        const json::Value* toe = v->find("toe_y");
        const json::Value* sh = v->find("shoulder_y");
        if (!toe || !toe->is_number() || !(toe->as_number() > 0)) c.bad("edr_tone_map.toe_y must be > 0");
        if (!sh || !sh->is_number() || !(sh->as_number() > toe->as_number())) c.bad("edr_tone_map.shoulder_y must be > toe_y");
        e.toe = toe->as_number();
        e.shoulder = sh->as_number();
        const json::Value* t = v->find("target_log2_y");
        if (!t) c.bad("edr_tone_map.target_log2_y is missing");
        e.target = vec(*t, 0, c, "edr_tone_map.target_log2_y");
        if (e.target.size() < 2) c.bad("edr_tone_map.target_log2_y needs at least 2 values");
        for (double x : e.target)
            if (!std::isfinite(x)) c.bad("edr_tone_map.target_log2_y must be finite");
        p.edr = std::move(e);
    }
    if (const json::Value* v = data.find("density_curves_model")) {
        if (!v->is_object()) c.bad("density_curves_model must be an object");
        if (const json::Value* t = v->find("model_type"); t && t->is_string()) p.model_type = t->as_string();
        auto part = [&](const char* k) {
            const json::Value* x = v->find(k);
            if (!x) c.bad(std::string("density_curves_model.") + k + " is missing");
            return mat_any(*x, c, k);
        };
        p.centers = part("centers");
        p.amplitudes = part("amplitudes");
        p.sigmas = part("sigmas");
        if (p.amplitudes.rows != p.centers.rows || p.amplitudes.cols != p.centers.cols ||
            p.sigmas.rows != p.centers.rows || p.sigmas.cols != p.centers.cols)
            c.bad("density_curves_model matrices differ in shape");
        p.has_model = true;
    }
    if (const json::Value* v = data.find("hanatos2025_adaptation_window_params")) {
        p.window = vec(*v, 0, c, "hanatos2025_adaptation_window_params");
        const size_t n = p.window.size();
        if (n != 0 && n != 4 && n != 8) c.bad("hanatos2025_adaptation_window_params must have 0, 4 or 8 values");
    }
}

void derive(Profile& p) {
    const size_t K = p.K();
    p.normalized = p.density_curves;
    for (size_t ch = 0; ch < 3; ++ch) {
        p.dmin[ch] = nanmin_strided(p.density_curves.v.data() + ch, K, 3);
        for (size_t k = 0; k < K; ++k) p.normalized(k, ch) = p.density_curves(k, ch) - p.dmin[ch];
        p.dmax[ch] = nanmax_strided(p.normalized.v.data() + ch, K, 3);
    }
}

void check_type(const Profile& p, const Ctx& c) {
    if (p.type != "negative" && p.type != "positive") c.bad("info.type '" + p.type + "' is not negative or positive");
}

}  // namespace

bool valid_stock_id(std::string_view id) {
    if (id.empty() || id.size() > 96) return false;
    for (char ch : id) {
        const bool ok = (ch >= 'A' && ch <= 'Z') || (ch >= 'a' && ch <= 'z') || (ch >= '0' && ch <= '9') ||
                        ch == '_' || ch == '-';
        if (!ok) return false;
    }
    return true;
}

std::shared_ptr<const Profile> load_profile(const std::filesystem::path& dir, std::string_view id) {
    Ctx c{std::string(id)};
    if (!valid_stock_id(id)) fail_user("invalid stock id '" + std::string(id) + "'");
    const json::Value doc = parse_file(dir / "profiles" / (std::string(id) + ".json"), c);
    if (!doc.is_object()) c.bad("the file is not a JSON object");
    auto p = std::make_shared<Profile>();
    p->id = std::string(id);
    const json::Value* df = doc.find("derived_from");
    const json::Value* info = nullptr;
    const json::Value* data = nullptr;
    json::Value base_doc;
    if (df && df->is_string()) {
        p->base_id = df->as_string();
        Ctx cb{std::string(id) + "' (alias of '" + p->base_id};
        if (!valid_stock_id(p->base_id)) cb.bad("invalid base stock id");
        base_doc = parse_file(dir / "profiles" / (p->base_id + ".json"), cb);
        if (!base_doc.is_object()) cb.bad("the base file is not a JSON object");
        if (const json::Value* d2 = base_doc.find("derived_from"); d2 && d2->is_string())
            cb.bad("an alias of an alias is refused");
        info = base_doc.find("info");
        data = base_doc.find("data");
        if (!info || !info->is_object()) cb.bad("'info' is missing");
        if (!data) cb.bad("'data' is missing");
        read_info(*info, *p);
        read_data(*data, *p, cb);
        if (const json::Value* ai = doc.find("info"); ai && ai->is_object()) read_info(*ai, *p);
    } else {
        info = doc.find("info");
        data = doc.find("data");
        if (!info || !info->is_object()) c.bad("'info' is missing");
        if (!data) c.bad("'data' is missing");
        read_info(*info, *p);
        read_data(*data, *p, c);
    }
    check_type(*p, c);
    derive(*p);
    return p;
}

// ---- Resources ------------------------------------------------------------------------------------

std::shared_ptr<Resources> Resources::load(const std::filesystem::path& dir) {
    std::error_code ec;
    if (!std::filesystem::is_directory(dir, ec)) fail_io("resources directory '" + dir.string() + "' does not exist");
    auto r = std::make_shared<Resources>();
    r->dir_ = dir;
    r->blob_ = Blob::open(dir / "spektralab_constants.bin");
    const std::filesystem::path fp = dir / "neutral_print_filters.json";
    if (std::filesystem::exists(fp, ec)) {
        std::ifstream f(fp, std::ios::binary);
        std::ostringstream ss;
        ss << f.rdbuf();
        try {
            r->filters_ = json::parse(ss.str());
        } catch (const json::ParseError& e) {
            fail_io(std::string("neutral_print_filters.json: ") + e.what());
        }
        if (!r->filters_.is_object()) fail_io("neutral_print_filters.json must be a JSON object");
    }
    // the print-preview table index (reference src/res/tables.cpp:80-115): optional; a malformed one fails
    const std::filesystem::path lp = dir / "print_luts.json";
    if (std::filesystem::exists(lp, ec)) {
        std::ifstream f(lp, std::ios::binary);
        std::ostringstream ss;
        ss << f.rdbuf();
        try {
            r->luts_ = json::parse(ss.str());
        } catch (const json::ParseError& e) {
            fail_io(std::string("print_luts.json: ") + e.what());
        }
        if (!r->luts_.is_object()) fail_io("print_luts.json: not an object");
        for (const auto& [stock, v] : r->luts_.as_object()) {
            auto bad = [&](const std::string& m) { fail_io("print_luts.json: '" + stock + "': " + m); };
            if (!v.is_object()) bad("not an object");
            const json::Value* pf = v.find("paired_film");
            if (!pf || !pf->is_string()) bad("missing paired_film");
            const json::Value* ls = v.find("lut_size");
            if (!ls || !ls->is_number()) bad("missing lut_size");
            const double sz = ls->as_number();
            if (!(sz > 1.0) || sz != std::floor(sz) || sz > 4096.0) bad("lut_size must be an integer > 1");
        }
        r->luts_present_ = true;
        r->lut_text_ = ss.str();
    }
    return r;
}

std::shared_ptr<const PrintLut> Resources::print_lut(std::string_view stock) const {
    {
        std::lock_guard<std::mutex> g(m_);
        auto it = lut_cache_.find(stock);
        if (it != lut_cache_.end()) return it->second;
    }
    if (!luts_present_) fail_user("no print-preview table index (print_luts.json) in the resources");
    const json::Value* v = luts_.find(std::string(stock));
    if (!v) {
        std::string list;
        for (const auto& [k, _] : luts_.as_object()) list += (list.empty() ? "" : ", ") + k;
        fail_user("no print-preview table for '" + std::string(stock) + "'; available: " + list);
    }
    auto t = std::make_shared<PrintLut>();
    t->stock = std::string(stock);
    t->paired_film = v->find("paired_film")->as_string();
    t->size = uint32_t(v->find("lut_size")->as_number());
    if (const json::Value* d = v->find("declared_pairing"); d && d->is_bool()) t->declared_pairing = d->as_bool();
    if (const json::Value* d = v->find("output_color_space"); d && d->is_string()) t->output_color_space = d->as_string();
    if (const json::Value* d = v->find("output_cctf_encoding"); d && d->is_bool()) t->output_cctf_encoding = d->as_bool();
    const uint32_t S = t->size;
    const std::string tname = "print_lut/" + std::string(stock), aname = "print_lut_axes/" + std::string(stock);
    const BlobEntry* te = blob_->find(tname);
    const BlobEntry* ae = blob_->find(aname);
    if (!te || te->dtype != 1 || te->ndim != 4 || te->dims[0] != S || te->dims[1] != S || te->dims[2] != S ||
        te->dims[3] != 3)
        fail_user("print-preview table '" + tname + "' is missing or has the wrong shape");
    if (!ae || ae->dtype != 1 || ae->ndim != 2 || ae->dims[0] != 3 || ae->dims[1] != S)
        fail_user("print-preview axes '" + aname + "' are missing or have the wrong shape");
    const std::vector<double> tv = blob_->f64(tname), av = blob_->f64(aname);  // binary32 widened exactly
    t->table.assign(tv.size(), 0.0f);
    for (size_t i = 0; i < tv.size(); ++i) t->table[i] = float(tv[i]);
    for (size_t c = 0; c < 3; ++c) {
        t->lo[c] = float(av[c * S]);
        t->hi[c] = float(av[c * S + S - 1]);
        if (!(t->hi[c] > t->lo[c])) fail_user("print-preview axes of '" + std::string(stock) + "' are not increasing");
    }
    std::lock_guard<std::mutex> g(m_);
    lut_cache_[std::string(stock)] = t;
    return t;
}

std::shared_ptr<const Profile> Resources::profile(std::string_view id) const {
    {
        std::lock_guard<std::mutex> g(m_);
        auto it = profiles_.find(id);
        if (it != profiles_.end()) return it->second;
    }
    std::shared_ptr<const Profile> p = load_profile(dir_, id);
    std::lock_guard<std::mutex> g(m_);
    profiles_[std::string(id)] = p;
    return p;
}

std::optional<Vec3> Resources::neutral_filters(std::string_view print, std::string_view illum,
                                               const Profile& film) const {
    auto leaf = [&](const std::string& film_id) -> std::optional<Vec3> {
        const json::Value* a = filters_.find(print);
        const json::Value* b = a ? a->find(illum) : nullptr;
        const json::Value* c = b ? b->find(film_id) : nullptr;
        if (!c || !c->is_array()) return std::nullopt;
        const auto& v = c->as_array();
        if (v.size() != 3 || !v[0].is_number() || !v[1].is_number() || !v[2].is_number()) return std::nullopt;
        return Vec3{v[0].as_number(), v[1].as_number(), v[2].as_number()};
    };
    if (auto r = leaf(film.id)) return r;
    if (!film.base_id.empty()) return leaf(film.base_id);
    return std::nullopt;
}

}  // namespace spkb
