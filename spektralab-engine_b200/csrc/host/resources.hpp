// The resources folder: the SPKR constants blob, named colour data, film/paper profiles and the
// neutral-filter database. Layout and rules: docs/RESOURCE_FORMAT.md of the reference engine.
// Everything here is binary64 set-up data; nothing runs on the device.
#pragma once

#include <array>
#include <cstdint>
#include <filesystem>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <string>
#include <string_view>
#include <vector>

#include "json.hpp"

namespace spkb {

using Spectrum = std::array<double, 81>;
using Mat3 = std::array<double, 9>;  // row-major: out_i = sum_j m[3i + j] x_j
using Vec3 = std::array<double, 3>;

// ---- the SPKR blob (docs/RESOURCE_FORMAT.md:213-246; reference src/res/blob.cpp:58-139) ----
struct BlobEntry {
    std::string name;
    uint32_t dtype = 0;  // 0 f64, 1 f32, 2 f16, 3 i32, 4 u8
    uint32_t ndim = 0;
    uint32_t dims[4] = {0, 0, 0, 0};
    uint64_t offset = 0, nbytes = 0;
    bool size_ok = false;
    uint64_t count() const;
};

class Blob {
public:
    static std::shared_ptr<const Blob> open(const std::filesystem::path& file);  // SPK_ERR_IO on failure
    ~Blob();
    const BlobEntry* find(std::string_view name) const;
    // Every value widened to binary64 (float16 decoded exactly); SPK_ERR_USER on a missing or bad entry.
    std::vector<double> f64(std::string_view name) const;
    size_t mapped_bytes() const { return size_; }

private:
    Blob() = default;
    const uint8_t* data_ = nullptr;
    size_t size_ = 0;
    std::map<std::string, BlobEntry, std::less<>> entries_;
};

// ---- colour (reference src/res/colour.cpp) ----
enum class Cctf : int { SRGB = 0, ProPhoto = 1, Adobe = 2, BT709 = 3, Identity = 4 };

struct ColourSpace {
    std::string name;
    Cctf cctf = Cctf::Identity;
    std::array<double, 6> primaries{};
    std::array<double, 2> whitepoint{};
    Mat3 rgb_to_xyz{}, xyz_to_rgb{};  // as stored in the blob, never re-derived
};

std::optional<Cctf> cctf_of(std::string_view name);  // the eight baked names
std::optional<ColourSpace> colour_space(const Blob& b, std::string_view name);
std::optional<Mat3> cat_matrix(const Blob& b, std::string_view name);
Spectrum blackbody(double kelvin);
std::optional<Spectrum> illuminant(const Blob& b, std::string_view name);  // normalised to mean 1
std::array<double, 2> chromaticity(const Blob& b, const Spectrum& s);

Mat3 mat3_mul(const Mat3& a, const Mat3& b);
Vec3 mat3_apply(const Mat3& m, const Vec3& v);
Mat3 mat3_inverse(const Mat3& m);  // adjugate with one reciprocal of the determinant
Vec3 xy_to_XYZ(const std::array<double, 2>& xy);
enum class Guard { Source, Target };
// Von Kries adaptation in the cone space `cone`; nullopt when the two whites are "allclose" (the
// guard compares against the source or the target white, as the caller states).
std::optional<Mat3> von_kries(const std::array<double, 2>& src, const std::array<double, 2>& dst, const Mat3& cone,
                              Guard g);

// ---- profiles (docs/RESOURCE_FORMAT.md:38-131; reference src/res/profile.cpp) ----
struct Mat {
    size_t rows = 0, cols = 0;
    std::vector<double> v;
    double operator()(size_t r, size_t c) const { return v[r * cols + c]; }
    double& operator()(size_t r, size_t c) { return v[r * cols + c]; }
};

struct Profile {
    std::string id, base_id;
    // info
    std::string type = "negative", support = "film", use = "still", antihalation = "weak";
    std::string reference_illuminant = "D55", viewing_illuminant = "D50";
    bool positive() const { return type == "positive"; }
    // data
    Mat log_sensitivity, channel_density;  // 81 x 3
    std::vector<double> base_density;      // 81
    std::vector<double> log_exposure;      // K
    Mat density_curves;                    // K x 3
    std::vector<double> layers;            // K x 3 x 3, [k][sublayer][channel]; empty when absent
    bool has_model = false;
    std::string model_type = "cdfs";
    Mat centers, amplitudes, sigmas;       // channels x layers
    std::vector<double> window;            // 0, 4 or 8 values
    // the EDR tone map of a paper (reference src/res/profile.hpp:69-76): log2 Y domain, toe and shoulder
    // luminances, the target curve in log2 Y
    struct Edr {
        double lo = 0.0, hi = 0.0, toe = 0.0, shoulder = 0.0;
        std::vector<double> target;
    };
    std::optional<Edr> edr;
    // derived at load
    std::array<double, 3> dmin{}, dmax{};
    Mat normalized;                        // K x 3: density - dmin
    size_t K() const { return log_exposure.size(); }
};

bool valid_stock_id(std::string_view id);
std::shared_ptr<const Profile> load_profile(const std::filesystem::path& dir, std::string_view id);

// ---- the resources folder ----
// A print-preview table (reference src/res/tables.hpp:48-62): S x S x S x 3 binary32, row-major
// [i][j][k][ch], over per-channel density axes lo..hi, with its print_luts.json entry.
struct PrintLut {
    std::string stock, paired_film, output_color_space;
    bool declared_pairing = false, output_cctf_encoding = true;
    uint32_t size = 0;
    std::vector<float> table;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

class Resources {
public:
    static std::shared_ptr<Resources> load(const std::filesystem::path& dir);
    const Blob& blob() const { return *blob_; }
    const std::filesystem::path& dir() const { return dir_; }
    // Cached per stock id; SPK_ERR_USER when the stock cannot be loaded.
    std::shared_ptr<const Profile> profile(std::string_view id) const;
    // The neutral filter pack for (print, illuminant, film), then the film's base id.
    std::optional<Vec3> neutral_filters(std::string_view print, std::string_view illum, const Profile& film) const;
    // print_luts.json as read ("{}" when absent), and one stock's table (cached; SPK_ERR_USER when the index,
    // the entry or its blob tables are missing or malformed).
    const std::string& print_lut_catalog() const { return lut_text_; }
    std::shared_ptr<const PrintLut> print_lut(std::string_view stock) const;

private:
    std::filesystem::path dir_;
    std::shared_ptr<const Blob> blob_;
    json::Value filters_;
    json::Value luts_;
    bool luts_present_ = false;
    std::string lut_text_ = "{}";
    mutable std::map<std::string, std::shared_ptr<const PrintLut>, std::less<>> lut_cache_;
    mutable std::mutex m_;
    mutable std::map<std::string, std::shared_ptr<const Profile>, std::less<>> profiles_;
};

// binary64 helpers with the reference's exact semantics (reference src/util/numeric.cpp)
double nanmin_strided(const double* p, size_t n, size_t stride);
double nanmax_strided(const double* p, size_t n, size_t stride);
double nanmean(const double* p, size_t n);
// Clamped piecewise-linear interpolation; NaN v gives NaN.
double interp(double v, const std::vector<double>& x, const std::vector<double>& y);
inline float f32(double x) { return static_cast<float>(x); }

}  // namespace spkb
