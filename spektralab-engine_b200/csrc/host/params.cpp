#include "params.hpp"

#include <cmath>
#include <cstdio>

#include "status.hpp"

namespace spkb {

namespace {

constexpr const char* kMethods[] = {"center_weighted", "average", "median", "balanced",
                                    "center", "protect_highlights", "protect_shadows"};

Field fl(const char* n, const char* path, double lo, double hi, double def, bool shoot, bool live = false) {
    return Field{n, path, FieldType::Float, true, lo, hi, json::Value(def), shoot, live};
}
Field in(const char* n, const char* path, double lo, double hi, double def, bool shoot) {
    return Field{n, path, FieldType::Int, true, lo, hi, json::Value(def), shoot, false};
}
Field bo(const char* n, const char* path, bool def, bool shoot) {
    return Field{n, path, FieldType::Bool, false, 0, 0, json::Value(def), shoot, false};
}
Field st(const char* n, const char* path, const char* def, bool shoot) {
    return Field{n, path, FieldType::Str, false, 0, 0, json::Value(def), shoot, false};
}

std::vector<Field> make_schema() {
    const bool S = true, Pr = false;
    return {
        st("film_stock", "film.info.stock", "kodak_portra_400", S),
        st("print_stock", "print.info.stock", "kodak_portra_endura", Pr),
        fl("exposure_compensation_ev", "camera.exposure_compensation_ev", -8, 8, 0, S),
        bo("auto_exposure", "camera.auto_exposure", true, S),
        st("auto_exposure_method", "camera.auto_exposure_method", "center_weighted", S),
        fl("film_format_mm", "camera.film_format_mm", 4, 200, 35, S),
        fl("lens_blur_um", "camera.lens_blur_um", 0, 200, 0, S),
        bo("halation_active", "film_render.halation.active", true, S),
        fl("halation_amount", "film_render.halation.halation_amount", 0, 4, 1, S),
        fl("halation_boost_ev", "film_render.halation.boost_ev", 0, 8, 0, S),
        bo("grain_active", "film_render.grain.active", true, S),
        bo("grain_sublayers_active", "film_render.grain.sublayers_active", true, S),
        bo("dir_couplers_active", "film_render.dir_couplers.active", true, S),
        fl("dir_couplers_amount", "film_render.dir_couplers.amount", 0, 4, 1, S),
        fl("density_curve_gamma", "film_render.density_curve_gamma", 0.2, 4, 1, S),
        st("input_color_space", "io.input_color_space", "ProPhoto RGB", S),
        bo("input_cctf_decoding", "io.input_cctf_decoding", false, S),
        fl("geometry_crop_x", "io.geometry.crop_x", 0, 1, 0, S),
        fl("geometry_crop_y", "io.geometry.crop_y", 0, 1, 0, S),
        fl("geometry_crop_w", "io.geometry.crop_w", 1e-4, 1, 1, S),
        fl("geometry_crop_h", "io.geometry.crop_h", 1e-4, 1, 1, S),
        fl("geometry_rotation_deg", "io.geometry.rotation_deg", -45, 45, 0, S),
        in("geometry_quarter_turns", "io.geometry.quarter_turns", 0, 3, 0, S),
        bo("geometry_flip_h", "io.geometry.flip_h", false, S),
        bo("geometry_flip_v", "io.geometry.flip_v", false, S),
        fl("print_exposure", "enlarger.print_exposure", 0.05, 20, 1, Pr, true),
        fl("m_filter_shift", "enlarger.m_filter_shift", -1, 1, 0, Pr, true),
        fl("y_filter_shift", "enlarger.y_filter_shift", -1, 1, 0, Pr, true),
        fl("c_filter_neutral", "enlarger.c_filter_neutral", 0, 200, 0, Pr),
        fl("m_filter_neutral", "enlarger.m_filter_neutral", 0, 200, 65, Pr),
        fl("y_filter_neutral", "enlarger.y_filter_neutral", 0, 200, 55, Pr),
        fl("preflash_exposure", "enlarger.preflash_exposure", 0, 1, 0, Pr, true),
        st("enlarger_illuminant", "enlarger.illuminant", "TH-KG3", Pr),
        bo("glare_active", "print_render.glare.active", true, Pr),
        bo("scanner_white_correction", "scanner.white_correction", false, Pr),
        bo("scanner_black_correction", "scanner.black_correction", false, Pr),
        fl("scanner_lens_blur", "scanner.lens_blur", 0, 20, 0, Pr),
        st("output_color_space", "io.output_color_space", "ProPhoto RGB", Pr),
        bo("output_cctf_encoding", "io.output_cctf_encoding", true, Pr),
        bo("scan_film", "io.scan_film", false, Pr),
        bo("extended_dynamic_range", "print_render.edr_enabled", false, Pr),
        fl("halation_scatter_amount", "film_render.halation.scatter_amount", 0, 1, 1, S),
        fl("grain_amount", "film_render.grain.amount", 0, 2, 1, S),
        fl("glare_amount", "print_render.glare.amount", 0, 30, 1, Pr),
        bo("antihalation_removed", "film_render.halation.antihalation_removed", false, S),
        fl("filter_shift_scale", "enlarger.filter_shift_scale", 1, 60, 1, Pr, true),
        fl("halation_headroom_ev", "film_render.halation.headroom_ev", 0, 8, 4, S),
        in("preview_long_edge", "io.preview_long_edge", 800, 8192, 1600, Pr),
    };
}

std::string fmt_f(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%f", v);
    return b;
}

const char* type_name(FieldType t) {
    switch (t) {
        case FieldType::Float: return "float";
        case FieldType::Int: return "int";
        case FieldType::Bool: return "bool";
        default: return "str";
    }
}

}  // namespace

const std::vector<Field>& schema() {
    static const std::vector<Field> s = make_schema();
    return s;
}

std::optional<size_t> find_field(std::string_view name) {
    const auto& s = schema();
    for (size_t i = 0; i < s.size(); ++i)
        if (name == s[i].name) return i;
    return std::nullopt;
}

const std::string& schema_json() {
    static const std::string text = [] {
        json::Array rows;
        for (const Field& f : schema()) {
            json::Value r;
            r["name"] = f.name;
            r["path"] = f.path;
            r["type"] = type_name(f.type);
            r["layer"] = f.shoot ? "shoot" : "print";
            r["default"] = f.def;
            r["live"] = f.live;
            if (f.has_range) r["range"] = json::Array{json::Value(f.lo), json::Value(f.hi)};
            rows.push_back(std::move(r));
        }
        json::Value doc;
        doc["schema_version"] = 1;
        doc["fields"] = std::move(rows);
        return json::write(doc);
    }();
    return text;
}

ParamSet::ParamSet() {
    for (const Field& f : schema()) v_.push_back(f.def);
}

json::Value ParamSet::to_json() const {
    json::Value o = json::Object{};
    const auto& s = schema();
    for (size_t i = 0; i < v_.size(); ++i) o[s[i].name] = v_[i];
    return o;
}

Delta validate_delta(std::string_view text, DeltaContext ctx) {
    Delta d;
    if (text.empty() && ctx == DeltaContext::Open) return d;
    json::Value doc;
    try {
        doc = json::parse(text);
    } catch (const json::ParseError& e) {
        fail_user(e.what());
    }
    if (!doc.is_object()) fail_user("params_delta must be an object");
    json::Object obj = doc.as_object();
    if (ctx == DeltaContext::Open) {
        if (auto it = obj.find("product_defaults"); it != obj.end()) {
            if (!it->second.is_bool()) fail_user("'product_defaults' expects bool");
            d.product_defaults = it->second.as_bool();
            obj.erase(it);
        }
    }
    for (const auto& [name, value] : obj) {
        const std::optional<size_t> id = find_field(name);
        if (!id) fail_user("unknown parameter '" + name + "'");
        const Field& f = schema()[*id];
        const bool type_ok = (f.type == FieldType::Float || f.type == FieldType::Int) ? value.is_number()
                             : f.type == FieldType::Bool                             ? value.is_bool()
                                                                                     : value.is_string();
        if (!type_ok) fail_user("'" + name + "' expects " + type_name(f.type));
        json::Value stored = value;
        if (*id == size_t(P::auto_exposure_method)) {
            bool ok = false;
            for (const char* m : kMethods) ok = ok || value.as_string() == m;
            if (!ok) {
                std::string list;
                for (const char* m : kMethods) list += (list.empty() ? "" : ", ") + std::string(m);
                fail_user("'auto_exposure_method' = '" + value.as_string() + "' is not one of " + list);
            }
        }
        if (f.type == FieldType::Float || f.type == FieldType::Int) {
            const double v = value.as_number();
            if (f.has_range) {
                if (!(v >= f.lo && v <= f.hi))
                    fail_user("'" + name + "'=" + fmt_f(v) + " is outside [" + fmt_f(f.lo) + ", " + fmt_f(f.hi) + "]");
            } else if (std::isnan(v)) {
                fail_user("'" + name + "' expects " + type_name(f.type) + ", not NaN");
            }
            if (f.type == FieldType::Int) stored = json::Value(std::round(v));
        }
        d.fields.emplace_back(*id, std::move(stored));
        if (*id == size_t(P::film_stock) || *id == size_t(P::print_stock)) d.has_stock = true;
        if (*id == size_t(P::preview_long_edge)) d.has_preview_long_edge = true;
        if (f.shoot) d.any_shoot = true;
        if (!f.live) d.any_rebuild = true;
    }
    if (d.has_stock) d.any_rebuild = true;
    return d;
}

void apply_delta(ParamSet& p, const Delta& d) {
    for (const auto& [id, v] : d.fields) p.set(id, v);
}

}  // namespace spkb
