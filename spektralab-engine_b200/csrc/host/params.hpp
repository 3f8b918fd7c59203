// The parameter schema (48 fields), the flat parameter values of a session, and delta validation.
// The field list, types, ranges, defaults, layers and live flags are part of the drop-in contract
// and equal the reference's (src/params/schema.cpp:51-115; docs/API_SPEC.md); validation follows
// src/params/delta.cpp:41-96: keys in bytewise order, first failure wins, SPK_ERR_USER.
#pragma once

#include <cstdint>
#include <memory>
#include <optional>
#include <string>
#include <string_view>
#include <vector>

#include "json.hpp"

namespace spkb {

enum class FieldType : uint8_t { Float, Int, Bool, Str };

struct Field {
    const char* name;
    const char* path;
    FieldType type;
    bool has_range;
    double lo, hi;
    json::Value def;
    bool shoot;  // layer "shoot" (film side) vs "print"
    bool live;
};

enum class P : uint16_t {
    film_stock, print_stock,
    exposure_compensation_ev, auto_exposure, auto_exposure_method, film_format_mm, lens_blur_um,
    halation_active, halation_amount, halation_boost_ev,
    grain_active, grain_sublayers_active,
    dir_couplers_active, dir_couplers_amount, density_curve_gamma,
    input_color_space, input_cctf_decoding,
    geometry_crop_x, geometry_crop_y, geometry_crop_w, geometry_crop_h, geometry_rotation_deg,
    geometry_quarter_turns, geometry_flip_h, geometry_flip_v,
    print_exposure, m_filter_shift, y_filter_shift, c_filter_neutral, m_filter_neutral, y_filter_neutral,
    preflash_exposure, enlarger_illuminant,
    glare_active, scanner_white_correction, scanner_black_correction, scanner_lens_blur,
    output_color_space, output_cctf_encoding, scan_film, extended_dynamic_range,
    halation_scatter_amount, grain_amount, glare_amount, antihalation_removed, filter_shift_scale,
    halation_headroom_ev, preview_long_edge,
    kCount
};
inline constexpr size_t kFieldCount = size_t(P::kCount);

const std::vector<Field>& schema();
std::optional<size_t> find_field(std::string_view name);
const std::string& schema_json();

class ParamSet {
public:
    ParamSet();  // schema defaults
    double f(P p) const { return v_[size_t(p)].as_number(); }
    int64_t i(P p) const { return int64_t(v_[size_t(p)].as_number()); }
    bool b(P p) const { return v_[size_t(p)].as_bool(); }
    const std::string& s(P p) const { return v_[size_t(p)].as_string(); }
    const json::Value& get(size_t id) const { return v_[id]; }
    void set(size_t id, json::Value v) { v_[id] = std::move(v); }
    void set(P p, json::Value v) { set(size_t(p), std::move(v)); }
    json::Value to_json() const;

private:
    std::vector<json::Value> v_;
};

struct Delta {
    std::vector<std::pair<size_t, json::Value>> fields;
    bool has_stock = false, any_shoot = false, any_rebuild = false, has_preview_long_edge = false;
    std::optional<bool> product_defaults;
};

enum class DeltaContext { Open, SetParams };
Delta validate_delta(std::string_view text, DeltaContext ctx);
void apply_delta(ParamSet& p, const Delta& d);

}  // namespace spkb
