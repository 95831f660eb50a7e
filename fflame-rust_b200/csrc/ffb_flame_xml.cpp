// ffb_flame_xml.cpp -- Apophysis / JWildfire `.flame` XML import: each
// <flame> (or layered <jwf-flame>) element becomes a `.fae` config (JSON),
// following src/flame_xml.rs:41-425 (attributes, unit conversions, the
// column-major `coefs` order, variation order = attribute order, finals
// attached to every normal, palette hex, Apophysis curves), 590-1014.
//
// Two differences, both because this build renders the 2-D path: the
// reference imports every flame in 3-D mode (flame_xml.rs:389); here the
// config is 2-D, and a flame whose camera leaves the plane (cam_pitch,
// cam_yaw, perspective, a z position, depth of field) is refused with the
// reason.  Variations outside this build's registry are carried into the
// config, where rendering refuses them by name.

#include "ffb_flame_xml.hpp"

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include "ffb_flame.hpp"
#include "ffb_json.hpp"

namespace ffb {

namespace {

[[noreturn]] void bad(const std::string& m) { throw std::runtime_error(m); }

// ------------------------------------------------------------------ XML --
struct XNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;   // in document order
    std::vector<XNode> kids;
    std::string text;
    bool empty = false;                                        // written <x .../>
    const std::string* attr(const char* k) const {
        for (auto& a : attrs) if (a.first == k) return &a.second;
        return nullptr;
    }
};

void utf8(std::string& o, uint32_t cp) {
    if (cp < 0x80) o.push_back((char)cp);
    else if (cp < 0x800) { o.push_back((char)(0xC0 | (cp >> 6))); o.push_back((char)(0x80 | (cp & 0x3F))); }
    else if (cp < 0x10000) {
        o.push_back((char)(0xE0 | (cp >> 12))); o.push_back((char)(0x80 | ((cp >> 6) & 0x3F))); o.push_back((char)(0x80 | (cp & 0x3F)));
    } else {
        o.push_back((char)(0xF0 | (cp >> 18))); o.push_back((char)(0x80 | ((cp >> 12) & 0x3F)));
        o.push_back((char)(0x80 | ((cp >> 6) & 0x3F))); o.push_back((char)(0x80 | (cp & 0x3F)));
    }
}

std::string unescape(const std::string& s) {
    std::string o;
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] != '&') { o.push_back(s[i]); continue; }
        const size_t e = s.find(';', i);
        if (e == std::string::npos) bad("XML: an unterminated entity");
        const std::string ent = s.substr(i + 1, e - i - 1);
        if (ent == "lt") o.push_back('<');
        else if (ent == "gt") o.push_back('>');
        else if (ent == "amp") o.push_back('&');
        else if (ent == "quot") o.push_back('"');
        else if (ent == "apos") o.push_back('\'');
        else if (!ent.empty() && ent[0] == '#') {
            const bool hex = ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X');
            utf8(o, (uint32_t)std::strtoul(ent.c_str() + (hex ? 2 : 1), nullptr, hex ? 16 : 10));
        } else bad("XML: unknown entity &" + ent + ";");
        i = e;
    }
    return o;
}

class XmlReader {
public:
    explicit XmlReader(const std::string& s) : s_(s) {}
    XNode document() {
        XNode root;
        root.name = "#document";
        parse_content(root);
        return root;
    }

private:
    const std::string& s_;
    size_t p_ = 0;

    bool starts(const char* t) const { return s_.compare(p_, std::strlen(t), t) == 0; }
    void skip_to(const char* t) {
        const size_t e = s_.find(t, p_);
        if (e == std::string::npos) bad(std::string("XML: missing ") + t);
        p_ = e + std::strlen(t);
    }
    void ws() { while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_; }
    std::string name() {
        const size_t b = p_;
        while (p_ < s_.size() && !std::isspace((unsigned char)s_[p_]) && s_[p_] != '>' && s_[p_] != '/' && s_[p_] != '=') ++p_;
        if (p_ == b) bad("XML: a name is missing at byte " + std::to_string(b));
        return s_.substr(b, p_ - b);
    }

    // Children of `node` until its end tag (or the end of the text at the root).
    void parse_content(XNode& node) {
        while (p_ < s_.size()) {
            if (s_[p_] != '<') {
                const size_t e = s_.find('<', p_);
                node.text += unescape(s_.substr(p_, (e == std::string::npos ? s_.size() : e) - p_));
                p_ = e == std::string::npos ? s_.size() : e;
                continue;
            }
            if (starts("<?")) { skip_to("?>"); continue; }
            if (starts("<!--")) { skip_to("-->"); continue; }
            if (starts("<![CDATA[")) {
                p_ += 9;
                const size_t e = s_.find("]]>", p_);
                if (e == std::string::npos) bad("XML: unterminated CDATA");
                node.text += s_.substr(p_, e - p_);
                p_ = e + 3;
                continue;
            }
            if (starts("<!")) {                                   // DOCTYPE, possibly with an internal subset
                int depth = 0;
                for (; p_ < s_.size(); ++p_) {
                    if (s_[p_] == '[') ++depth;
                    else if (s_[p_] == ']') --depth;
                    else if (s_[p_] == '>' && depth <= 0) { ++p_; break; }
                }
                continue;
            }
            if (starts("</")) {
                p_ += 2;
                const std::string n = name();
                ws();
                if (p_ >= s_.size() || s_[p_] != '>') bad("XML: a malformed end tag");
                ++p_;
                if (n != node.name) bad("XML: </" + n + "> closes <" + node.name + ">");
                return;
            }
            ++p_;
            XNode kid;
            kid.name = name();
            for (;;) {
                ws();
                if (p_ >= s_.size()) bad("XML: an unterminated tag <" + kid.name + ">");
                if (s_[p_] == '/') {
                    if (p_ + 1 >= s_.size() || s_[p_ + 1] != '>') bad("XML: a malformed empty tag");
                    p_ += 2;
                    kid.empty = true;
                    break;
                }
                if (s_[p_] == '>') { ++p_; parse_content(kid); break; }
                const std::string k = name();
                ws();
                if (p_ >= s_.size() || s_[p_] != '=') bad("XML: attribute " + k + " has no value");
                ++p_;
                ws();
                if (p_ >= s_.size() || (s_[p_] != '"' && s_[p_] != '\'')) bad("XML: attribute " + k + " is not quoted");
                const char q = s_[p_++];
                const size_t e = s_.find(q, p_);
                if (e == std::string::npos) bad("XML: attribute " + k + " is not terminated");
                kid.attrs.push_back({k, unescape(s_.substr(p_, e - p_))});
                p_ = e + 1;
            }
            node.kids.push_back(std::move(kid));
        }
        if (node.name != "#document") bad("XML: <" + node.name + "> is not closed");
    }
};

// -------------------------------------------------------------- values --
bool num(const std::string& v, float& out) {
    const char* b = v.c_str();
    while (*b && std::isspace((unsigned char)*b)) ++b;
    char* e = nullptr;
    const float x = std::strtof(b, &e);
    if (e == b) return false;
    while (*e && std::isspace((unsigned char)*e)) ++e;
    if (*e) return false;
    out = x;
    return true;
}
float num_or(const std::string* v, float d) {
    float x;
    return v && num(*v, x) ? x : d;
}
std::vector<float> nums(const std::string& v) {
    std::vector<float> o;
    const char* p = v.c_str();
    while (*p) {
        char* e = nullptr;
        const float x = std::strtof(p, &e);
        if (e == p) { ++p; continue; }
        o.push_back(x);
        p = e;
    }
    return o;
}
std::string f(float v) {
    char b[48];
    std::snprintf(b, sizeof b, "%.9g", (double)v);
    return b;
}

// Attributes of an <xform> that are not variations (Apophysis 7X and
// JWildfire write these; the reference's parser skips them because its
// registry does not know them as variations).
bool not_a_variation(const std::string& k) {
    static const char* const names[] = {
        "weight", "color", "symmetry", "color_speed", "coefs", "post", "opacity", "chaos", "animate", "name",
        "var_color", "plotmode", "mod_gamma", "mod_gamma_speed", "mod_contrast",
        "mod_contrast_speed", "mod_saturation", "mod_saturation_speed", "mod_hue", "mod_hue_speed", "material",
        "material_speed", "color_type", "target_color", "drawMode", "draw_mode", "visible", "xyCoefs", "yzCoefs",
        "zxCoefs", "xyPost", "yzPost", "zxPost", "dc_weight"};
    for (const char* n : names) if (k == n) return true;
    return k.rfind("motion_", 0) == 0 || k.rfind("subflame_wf_flame", 0) == 0 ||
           (k.size() > 12 && k.compare(k.size() - 12, 12, "_fx_priority") == 0);
}

// The canonical name of a variation of this build's registry (aliases
// resolved: cylinder_apo is cylinder, variations/defs/advanced.rs:670).
const VarDef* registry_var(const std::string& k) {
    if (k == "cylinder_apo") return registry_find("cylinder");
    return registry_find(k);
}

struct XformOut {
    float a = 1, b = 0, c = 0, d = 1, e = 0, fc = 0;
    bool post = false;
    float pa = 1, pb = 0, pc = 0, pd = 1, pe = 0, pf = 0;
    float weight = 1, color = 0.5f, speed = 0, opacity = 1;
    bool has_dc = false;
    float direct_color = 1;                                   // pluginColor (transforms.rs:411-419)
    std::vector<std::pair<std::string, float>> vars;          // canonical name, summed weight, first-seen order
    std::vector<std::pair<std::string, float>> params;        // "name.param", value
    std::vector<float> chaos;
};

void coefs(const std::string& v, float& a, float& b, float& c, float& d, float& e, float& ff) {
    // "a c b d e f": Apophysis writes the matrix column-major (flame_xml.rs:640-651).
    const std::vector<float> p = nums(v);
    if (p.size() < 6) return;
    a = p[0]; c = p[1]; b = p[2]; d = p[3]; e = p[4]; ff = p[5];
}

XformOut parse_xform(const XNode& x, bool is_final) {
    XformOut t;
    std::vector<std::pair<std::string, float>> pending;       // params, applied after the variations are known
    for (auto& [k, v] : x.attrs) {
        if (k == "weight") { if (!is_final) t.weight = num_or(&v, 1.0f); }
        else if (k == "color") { const std::vector<float> p = nums(v); if (!p.empty()) t.color = p[0]; }
        else if (k == "color_speed" || k == "symmetry") t.speed = num_or(&v, 0.0f);
        else if (k == "opacity") { if (!is_final) t.opacity = num_or(&v, 1.0f); }
        else if (k == "pluginColor" || k == "plugin_color") { t.has_dc = true; t.direct_color = num_or(&v, 0.0f); }
        else if (k == "coefs") coefs(v, t.a, t.b, t.c, t.d, t.e, t.fc);
        else if (k == "post") {
            if (nums(v).size() >= 6) { t.post = true; coefs(v, t.pa, t.pb, t.pc, t.pd, t.pe, t.pf); }
        } else if (k == "chaos") { if (!is_final) t.chaos = nums(v); }
        else if (not_a_variation(k)) continue;
        else {
            float val;
            if (!num(v, val)) continue;
            const VarDef* vd = registry_var(k);
            std::string var;
            if (vd) var = vd->name;
            else {
                // "name_param" of a registry variation (flame_xml.rs:986-1010).
                bool is_param = false;
                for (size_t u = k.rfind('_'); u != std::string::npos && u > 0; u = k.rfind('_', u - 1)) {
                    const VarDef* pv = registry_var(k.substr(0, u));
                    if (!pv) continue;
                    const std::string pn = k.substr(u + 1);
                    for (int q = 0; q < pv->nparams; ++q)
                        if (pn == pv->pname[q]) {
                            // The .flame's units (flame_xml.rs:957-974): radial_blur's
                            // angle is in half turns, the config's in degrees.
                            const float v = (std::string(pv->name) == "radial_blur" && pn == "angle") ? val * 180.0f : val;
                            pending.push_back({std::string(pv->name) + "." + pn, v});
                            is_param = true;
                        }
                    if (is_param) break;
                }
                if (is_param) continue;
                // A parameter of a variation this build lacks: "name_param"
                // where `name` is another attribute of this xform.
                for (size_t u = k.rfind('_'); u != std::string::npos && u > 0 && !is_param; u = k.rfind('_', u - 1)) {
                    const std::string pre = k.substr(0, u);
                    if (not_a_variation(pre)) continue;
                    for (auto& kv : x.attrs)
                        if (kv.first == pre) { pending.push_back({pre + "." + k.substr(u + 1), val}); is_param = true; break; }
                }
                if (is_param) continue;
                var = k;                                      // a variation this build lacks: kept, refused at render
            }
            if (val == 0.0f) continue;
            auto it = std::find_if(t.vars.begin(), t.vars.end(), [&](auto& p) { return p.first == var; });
            if (it == t.vars.end()) t.vars.push_back({var, val});
            else it->second += val;
        }
    }
    t.params = pending;
    return t;
}

std::string xform_json(const XformOut& t, bool is_final, int n_finals) {
    JsonWriter w;
    w.begin();
    w.raw("a", f(t.a)).raw("b", f(t.b)).raw("c", f(t.c)).raw("d", f(t.d)).raw("e", f(t.e)).raw("f", f(t.fc));
    if (t.post) {
        w.boolean("post_affine_enabled", true);
        w.raw("post_a", f(t.pa)).raw("post_b", f(t.pb)).raw("post_c", f(t.pc)).raw("post_d", f(t.pd))
         .raw("post_e", f(t.pe)).raw("post_f", f(t.pf));
    }
    // A final's weight and opacity are not read from the XML; the
    // reference's config carries its defaults (transforms.rs:497-505).
    w.raw("weight", f(is_final ? 1.0f : t.weight)).raw("opacity", f(is_final ? 1.0f : t.opacity));
    w.raw("color", f(t.color)).raw("color_speed", f(t.speed));
    if (t.has_dc) w.raw("direct_color", f(t.direct_color));
    std::string vars = "{", order = "[", prm = "{";
    for (size_t i = 0; i < t.vars.size(); ++i) {
        vars += (i ? "," : "") + JsonWriter::quote(t.vars[i].first) + ":" + f(t.vars[i].second);
        order += (i ? "," : "") + JsonWriter::quote(t.vars[i].first);
    }
    for (size_t i = 0; i < t.params.size(); ++i) prm += (i ? "," : "") + JsonWriter::quote(t.params[i].first) + ":" + f(t.params[i].second);
    w.raw("variations", vars + "}").raw("variation_order", order + "]");
    if (!t.params.empty()) w.raw("variation_params", prm + "}");
    if (!is_final && n_finals > 0) {
        std::string att = "[";
        for (int i = 0; i < n_finals; ++i) att += (i ? "," : "") + std::to_string(i);
        w.raw("final_attachments", att + "]");
    }
    w.end();
    return w.s();
}

// Apophysis curves: 48 floats, the first 12 the overall curve as a rational
// cubic Bezier of 4 (x, y, weight) points, sampled at t = 1/4, 1/2, 3/4
// between the end points (flame_xml.rs:1084-1150).
std::string curve_json(const std::vector<float>& d) {
    std::vector<std::pair<float, float>> pts = {{0.0f, 0.0f}};
    if (d.size() == 48) {
        for (float t : {0.25f, 0.5f, 0.75f}) {
            const float s = 1.0f - t, s2 = s * s, s3 = s2 * s, t2 = t * t, t3 = t2 * t;
            const float b0 = d[2] * s3, b1 = d[5] * 3.0f * s2 * t, b2 = d[8] * 3.0f * s * t2, b3 = d[11] * t3;
            const float nx = b0 * d[0] + b1 * d[3] + b2 * d[6] + b3 * d[9];
            const float ny = b0 * d[1] + b1 * d[4] + b2 * d[7] + b3 * d[10];
            const float den = b0 + b1 + b2 + b3;
            if (std::fabs(den) < 1e-10f) continue;
            pts.push_back({nx / den, ny / den});
        }
    }
    pts.push_back({1.0f, 1.0f});
    std::stable_sort(pts.begin(), pts.end(), [](auto& a, auto& b) { return a.first < b.first; });
    std::string o = "{\"points\":[";
    for (size_t i = 0; i < pts.size(); ++i) o += (i ? "," : "") + std::string("{\"x\":") + f(pts[i].first) + ",\"y\":" + f(pts[i].second) + "}";
    return o + "]}";
}

// <palette count="256" format="RGB">hex</palette>: 256 colours, 6 hex digits
// each, as stops at i/255 (flame_xml.rs:1014-1082); written as the
// config's `indexed_colors`, which reads back to the same stops.
std::string palette_json(const XNode& p) {
    std::string hex;
    for (char ch : p.text) if (!std::isspace((unsigned char)ch)) hex.push_back(ch);
    if (hex.size() < 1536) bad("Invalid palette data: expected 1536 hex characters, got " + std::to_string(hex.size()));
    std::string cols;
    for (int i = 0; i < 256; ++i) {
        const std::string c = hex.substr((size_t)i * 6, 6);
        for (char ch : c) if (!std::isxdigit((unsigned char)ch)) bad("Invalid palette data: `" + c + "` is not hex");
        if (i) cols += ",";
        for (char ch : c) cols.push_back((char)std::toupper((unsigned char)ch));
    }
    return "{\"name\":\"Imported from Apophysis\",\"indexed_colors\":\"" + cols + "\"}";
}

void collect(const XNode& n, std::vector<const XNode*>& out) {
    for (auto& k : n.kids) {
        // <flame> written as an empty element carries no transforms; the
        // reference reads only elements with content (flame_xml.rs:50-58).
        if ((k.name == "flame" || k.name == "jwf-flame") && !k.empty) out.push_back(&k);
        else collect(k, out);
    }
}

std::string flame_json(const XNode& fl) {
    auto A = [&](const char* k) { return fl.attr(k); };
    std::string name = A("name") ? *A("name") : "Untitled";
    float sw = 1920, sh = 1080;
    if (auto* v = A("size")) { auto p = nums(*v); if (p.size() == 2) { sw = p[0]; sh = p[1]; } }
    float cx = 0, cy = 0;
    if (auto* v = A("center")) { auto p = nums(*v); if (p.size() == 2) { cx = p[0]; cy = p[1]; } }
    const float scale = num_or(A("scale"), 100.0f), rotate = num_or(A("rotate"), 0.0f);
    float bg[3] = {0, 0, 0};
    if (auto* v = A("background")) { auto p = nums(*v); if (p.size() == 3) for (int i = 0; i < 3; ++i) bg[i] = p[i] / 255.0f; }
    const float brightness = num_or(A("brightness"), 1.0f), gamma = num_or(A("gamma"), 2.2f);
    const float vibrancy = num_or(A("vibrancy"), 1.0f), gthr = num_or(A("gamma_threshold"), 0.0025f);
    const float filter = num_or(A("filter"), 0.0f), cam_zoom = num_or(A("cam_zoom"), 1.0f);
    const float saturation = num_or(A("saturation"), 1.0f), white = num_or(A("white_level"), 200.0f);
    // A camera out of the plane has no 2-D rendering.
    for (const char* k : {"cam_pitch", "cam_yaw", "cam_perspective", "cam_persp", "cam_zpos", "cam_pos_x", "cam_pos_y",
                          "cam_pos_z", "cam_dof", "cam_roll"})
        if (std::fabs(num_or(A(k), 0.0f)) > 1e-4f)
            bad("flame `" + name + "` uses a 3-D camera (" + k + "); this build renders 2-D flames");
    std::string sym;
    if (auto* v = A("post_symmetry_type")) {
        std::string t = *v;
        for (auto& ch : t) ch = (char)std::toupper((unsigned char)ch);
        // The axis names swap on the wire (transforms.rs:2116-2146).
        const char* ty = t == "X_AXIS" ? "yaxis" : t == "Y_AXIS" ? "xaxis" : t == "POINT" ? "point" : "none";
        const float order = num_or(A("post_symmetry_order"), 3.0f);
        const float scx = A("post_symmetry_centre_x") ? num_or(A("post_symmetry_centre_x"), 0) : num_or(A("post_symmetry_center_x"), 0);
        const float scy = A("post_symmetry_centre_y") ? num_or(A("post_symmetry_centre_y"), 0) : num_or(A("post_symmetry_center_y"), 0);
        sym = std::string("{\"ty\":\"") + ty + "\",\"order\":" + std::to_string((int)std::max(order, 0.0f)) + ",\"center_x\":" + f(scx) +
              ",\"center_y\":" + f(scy) + ",\"distance\":" + f(num_or(A("post_symmetry_distance"), 1.25f)) +
              ",\"rotation_deg\":" + f(num_or(A("post_symmetry_rotation"), 6.0f)) + "}";
    }
    std::vector<float> curves;
    if (auto* v = A("curves")) curves = nums(*v);
    if (curves.size() != 48) curves.clear();
    int solo = -1;
    if (auto* v = A("soloxform")) { float s; if (num(*v, s) && s >= 0) solo = (int)s; }

    // Transforms and the palette, in document order at any depth below the
    // flame element, except inside the second and later <layer> of a
    // <jwf-flame> (flame_xml.rs:286-330); <bgxform> is not an xform, and
    // of several palettes the last is kept.
    std::vector<XformOut> xfs, fins;
    const XNode* palette = nullptr;
    int layers_seen = 0;
    std::function<void(const XNode&)> walk = [&](const XNode& n) {
        for (auto& k : n.kids) {
            if (k.name == "layer") {
                if (layers_seen++ == 0) walk(k);
                continue;
            }
            if (k.name == "palette") { palette = &k; continue; }
            if (k.name == "xform") xfs.push_back(parse_xform(k, false));
            else if (k.name == "finalxform") fins.push_back(parse_xform(k, true));
            walk(k);
        }
    };
    walk(fl);

    JsonWriter fw;
    fw.begin().str("name", name);
    std::string ts = "[";
    for (size_t i = 0; i < xfs.size(); ++i) ts += (i ? "," : "") + xform_json(xfs[i], false, (int)fins.size());
    fw.raw("transforms", ts + "]");
    if (!fins.empty()) {
        std::string fs = "[";
        for (size_t i = 0; i < fins.size(); ++i) fs += (i ? "," : "") + xform_json(fins[i], true, 0);
        fw.raw("final_transforms", fs + "]");
    }
    bool any_chaos = false;
    for (auto& x : xfs) any_chaos |= !x.chaos.empty();
    if (any_chaos) {                                       // rows default to 1 (flame_xml.rs:355-375)
        std::string m = "[";
        for (size_t i = 0; i < xfs.size(); ++i) {
            m += i ? ",[" : "[";
            for (size_t j = 0; j < xfs.size(); ++j) m += (j ? "," : "") + f(j < xfs[i].chaos.size() ? xfs[i].chaos[j] : 1.0f);
            m += "]";
        }
        fw.raw("xaos", m + "]");
    }
    if (solo >= 0) fw.num("solo_transform", solo);
    if (!sym.empty()) fw.raw("post_symmetry", sym);
    fw.end();

    JsonWriter w;
    w.begin();
    w.str("name", name).str("render_mode", "TwoD").raw("flame", fw.s());
    w.raw("image_size", "[" + std::to_string((long long)sw) + "," + std::to_string((long long)sh) + "]");
    // scale is pixels a unit: 200 is zoom 1 (flame_xml.rs:414-421); rotate is degrees.
    w.raw("zoom", f((scale / 200.0f) * cam_zoom)).raw("pan_x", f(cx)).raw("pan_y", f(cy));
    w.raw("rotation", f(rotate * 3.14159265358979323846f / 180.0f));
    w.raw("background_color", "[" + f(bg[0]) + "," + f(bg[1]) + "," + f(bg[2]) + "]");
    w.raw("brightness", f(brightness)).raw("gamma", f(gamma)).raw("vibrancy", f(vibrancy));
    w.raw("gamma_threshold", f(gthr * 2000.0f + 50.0f));           // Apophysis scale -> ours (flame_xml.rs:426-432)
    w.raw("white_level", f(white)).raw("saturation", f(saturation)).raw("filter_radius", f(filter));
    w.str("tonemap_mode", "Logarithmic").str("highlight_mode", "Clip").boolean("use_curve", true).raw("exposure", "1");
    w.raw("tonemap_curve", curve_json(curves));
    w.raw("density_scale", "1").raw("speed_factor", "1").num("max_iterations", 1e9).boolean("deterministic_rng", false);
    w.str("color_mode", "Palette");
    if (palette) w.raw("palette", palette_json(*palette));
    w.end();
    return w.s();
}

}  // namespace

std::vector<std::string> flame_xml_import(const std::string& xml) {
    XmlReader rd(xml);
    const XNode doc = rd.document();
    std::vector<const XNode*> flames;
    collect(doc, flames);
    if (flames.empty()) bad("No <flame> or <jwf-flame> elements found in XML");
    std::vector<std::string> out;
    for (const XNode* fl : flames) out.push_back(flame_json(*fl));
    return out;
}

}  // namespace ffb
